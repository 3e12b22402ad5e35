// Periodic 3x3 convolutions of the correction network on the sm_100a tensor cores (tcgen05.mma,
// BF16 operands, FP32 accumulators in TMEM), forward and backward.
//
// Semantics follow the reference's PeriodicConv (surrogate/models.py:16-29): wrap-pad by 1, then a
// VALID 3x3 cross-correlation with weight (c_out, c_in, 3, 3) and a bias; the hidden activation is
// jax.nn.gelu's default tanh approximation (models.py:43-44).
//
// Layout: activations NHWC bf16 with the channel count padded to 16 or 32; weights packed for the
// MMA B operand as [shift = ky*3+kx][c_in/8][c_out][8] (K-major core matrices, 16 bytes per row).
//
// Forward (implicit GEMM, M = pixels, N = c_out, K = 9 * c_in): a CTA owns 256 output pixels
// (256/W image rows).  It stages the (rows + 2) input rows three times, shifted in x by kx - 1 with
// periodic wrap, in the K-major layout [kx][c_in/8][pixel][8]; then for every shift (ky, kx) the A
// operand of the 128-pixel M-tile is that copy started ky rows further -- a plain descriptor offset,
// no im2col buffer.  Two M-tiles x 9 shifts x (c_in/16) K-steps of tcgen05.mma (M=128, K=16) go to
// TMEM; the epilogue (tcgen05.ld, one accumulator row per thread) adds the bias and applies GELU, or
// for the backward-data pass multiplies by GELU'(pre-activation of the layer below).
// Backward data is the same kernel with the weights transposed (c_in <-> c_out) and flipped.
// Image widths >= 64 use a row kernel that stages each input row once and takes the x-shifts as
// descriptor offsets of M = 64 tiles (conv3x3_rows_kernel).
// Backward weights (per x-shift: M = 3 * c_in rows (ky, c_in), N = c_out, K = pixels): per image row
// the MMAs read the staged input rows and output-gradient row in place as MN-major operands and
// accumulate in TMEM over the CTA's rows; per-CTA partial sums are reduced in a fixed order
// (deterministic).
#include <cuda_bf16.h>
#include <cuda_runtime.h>

#include <algorithm>
#include <cstdint>
#include <cstdlib>

#include "../../include/fvnet.h"
#include "tc_sm100.cuh"

int fv_internal_set_error(int code, const char* msg);

namespace fvnet {

constexpr int NT = 128;
constexpr float kGeluC0 = 0.7978845608028654f;  // sqrt(2/pi)
constexpr float kGeluC1 = 0.044715f;

__device__ __forceinline__ float gelu_tanh(float z) {
    const float t = tanhf(kGeluC0 * (z + kGeluC1 * z * z * z));
    return 0.5f * z * (1.0f + t);
}
__device__ __forceinline__ float gelu_tanh_grad(float z) {
    const float t = tanhf(kGeluC0 * (z + kGeluC1 * z * z * z));
    return 0.5f * (1.0f + t) + 0.5f * z * (1.0f - t * t) * kGeluC0 * (1.0f + 3.0f * kGeluC1 * z * z);
}

struct ConvArgs {
    const uint4* X;       // [B][H][W][CIN] bf16, as 16-byte chunks
    const uint4* Wb;      // packed weights [9][CIN/8][COUT][8] bf16
    const float* bias;    // [COUT] (forward modes)
    const __nv_bfloat16* Zprev;  // [B][H][W][COUT] (mode BWD_GELU)
    __nv_bfloat16* Z;     // [B][H][W][COUT] pre-activation (mode HIDDEN)
    __nv_bfloat16* A;     // [B][H][W][COUT] activation (HIDDEN) or input gradient (BWD_*)
    float* out4;          // [B][H][W][4] (mode OUTPUT)
    int B, H, W;
    int* err;
};

__device__ __forceinline__ uint4 pack8(const float* v) {
    __nv_bfloat162 p0 = __floats2bfloat162_rn(v[0], v[1]), p1 = __floats2bfloat162_rn(v[2], v[3]);
    __nv_bfloat162 p2 = __floats2bfloat162_rn(v[4], v[5]), p3 = __floats2bfloat162_rn(v[6], v[7]);
    uint4 u;
    u.x = *reinterpret_cast<uint32_t*>(&p0);
    u.y = *reinterpret_cast<uint32_t*>(&p1);
    u.z = *reinterpret_cast<uint32_t*>(&p2);
    u.w = *reinterpret_cast<uint32_t*>(&p3);
    return u;
}

// Staging planes ([kx][cc] copies of the TR + 2 rows) are NPIX + 2 chunks apart: the 32-byte pad puts
// the four channel chunks of one pixel, stored by neighbouring threads, in different bank groups.
__host__ __device__ constexpr int conv_plane(int W) { return (256 / W + 2) * W + 2; }
__host__ __device__ constexpr size_t conv_smem_bytes(int cin, int cout, int W) {
    return size_t(3) * (cin / 8) * conv_plane(W) * 16 + size_t(9) * (cin / 8) * cout * 16 + 64;
}

template <int CIN, int COUT, int MODE>
__global__ void __launch_bounds__(NT) conv3x3_kernel(ConvArgs a) {
    constexpr int CC = CIN / 8;
    extern __shared__ __align__(1024) unsigned char smem[];
    const int W = a.W, H = a.H;
    const int TR = 256 / W, PS = conv_plane(W);
    uint4* Xc = reinterpret_cast<uint4*>(smem);                  // [3][CC][PS] (NPIX used + pad)
    uint4* Wt = Xc + size_t(3) * CC * PS;                        // [9][CC][COUT]
    uint64_t* bar = reinterpret_cast<uint64_t*>(Wt + 9 * CC * COUT);
    uint32_t* tslot = reinterpret_cast<uint32_t*>(bar + 1);
    const int tid = threadIdx.x, warp = tid >> 5, lane = tid & 31;
    const int n = blockIdx.y, y0 = blockIdx.x * TR;
    constexpr uint32_t kCols = (2 * COUT) < 32 ? 32 : 2 * COUT;

    if (warp == 0) tc::tmem_alloc(tslot, kCols);
    if (tid == 0) {
        tc::mbar_init(bar, 1);
        tc::fence_mbar_init();
    }
    // stage three x-shifted copies of rows y0-1 .. y0+TR (periodic in x and y); unrolled so that
    // several global loads are in flight before their stores
#pragma unroll 4
    for (int e = tid; e < (TR + 2) * W * CC; e += NT) {
        const int cc = e % CC, t = e / CC, x = t % W, r = t / W;
        const int y = (y0 - 1 + r + H) % H;
        const uint4 v = a.X[(size_t(n * H + y) * W + x) * CC + cc];
#pragma unroll
        for (int kx = 0; kx < 3; ++kx) {
            const int xd = (x - kx + 1 + W) % W;
            Xc[(size_t(kx) * CC + cc) * PS + r * W + xd] = v;
        }
    }
    for (int e = tid; e < 9 * CC * COUT; e += NT) Wt[e] = a.Wb[e];
    tc::fence_proxy_async_smem();
    tc::fence_before_sync();
    __syncthreads();
    tc::fence_after_sync();
    const uint32_t tmem = *tslot;

    if (tid == 0) {
        constexpr uint32_t idesc = tc::idesc_bf16_f32(128, COUT);
        const uint32_t xb = tc::smem_addr(Xc), wb = tc::smem_addr(Wt);
        const uint32_t lbo_a = uint32_t(PS) * 16, lbo_b = COUT * 16;
        for (int mt = 0; mt < 2; ++mt)
            for (int sh = 0; sh < 9; ++sh) {
                const int ky = sh / 3, kx = sh % 3;
                for (int s = 0; s < CIN / 16; ++s) {
                    const uint32_t aa = xb + ((kx * CC + 2 * s) * PS + mt * 128 + ky * W) * 16;
                    const uint32_t ba = wb + (sh * CC + 2 * s) * COUT * 16;
                    tc::mma_bf16(tmem + mt * COUT, tc::smem_desc(aa, lbo_a, 128), tc::smem_desc(ba, lbo_b, 128), idesc,
                                 (sh | s) != 0);
                }
            }
        tc::mma_commit(bar);
    }
    const bool ok = tc::mbar_wait_bounded(bar, 0, a.err);
    tc::fence_after_sync();
    if (ok) {
        for (int mt = 0; mt < 2; ++mt) {
            float acc[32];
            const uint32_t taddr = tmem + (uint32_t(warp * 32) << 16) + mt * COUT;
            if constexpr (COUT == 32) tc::tmem_ld_32x32(taddr, acc);
            else tc::tmem_ld_32x16(taddr, acc);
            const int m = mt * 128 + warp * 32 + lane;
            const int r = m / W, x = m % W;
            const size_t gp = size_t(n * H + y0 + r) * W + x;
            if constexpr (MODE == FVNET_CONV_HIDDEN) {
                float z[COUT], g[COUT];
#pragma unroll
                for (int c = 0; c < COUT; ++c) {
                    z[c] = acc[c] + a.bias[c];
                    g[c] = gelu_tanh(z[c]);
                }
                uint4* Zo = reinterpret_cast<uint4*>(a.Z + gp * COUT);
                uint4* Ao = reinterpret_cast<uint4*>(a.A + gp * COUT);
#pragma unroll
                for (int q = 0; q < COUT / 8; ++q) {
                    Zo[q] = pack8(z + 8 * q);
                    Ao[q] = pack8(g + 8 * q);
                }
            } else if constexpr (MODE == FVNET_CONV_OUTPUT) {
                float4 o = make_float4(acc[0] + a.bias[0], acc[1] + a.bias[1], acc[2] + a.bias[2], acc[3] + a.bias[3]);
                reinterpret_cast<float4*>(a.out4)[gp] = o;
            } else {
                float d[COUT];
                const uint4* Zp = reinterpret_cast<const uint4*>(a.Zprev + gp * COUT);
#pragma unroll
                for (int q = 0; q < COUT / 8; ++q) {
                    const uint4 u = Zp[q];
                    const __nv_bfloat16* zb = reinterpret_cast<const __nv_bfloat16*>(&u);
#pragma unroll
                    for (int j = 0; j < 8; ++j) {
                        const float gz = (MODE == FVNET_CONV_BWD_GELU) ? gelu_tanh_grad(__bfloat162float(zb[j])) : 1.0f;
                        d[8 * q + j] = acc[8 * q + j] * gz;
                    }
                }
                uint4* Ao = reinterpret_cast<uint4*>(a.A + gp * COUT);
#pragma unroll
                for (int q = 0; q < COUT / 8; ++q) Ao[q] = pack8(d + 8 * q);
            }
        }
    }
    tc::fence_before_sync();
    __syncthreads();
    if (warp == 0) tc::tmem_dealloc(tmem, kCols);
}

// ---- forward / backward data, one staged copy (image widths >= 64) -------------------------------
// The same implicit GEMM with a quarter of the shared memory, so that more CTAs (warps) fit per SM:
// the rows y0-1 .. y0+TR are staged once, each row padded with its periodic neighbours
// ([cc][row][x = -1, 0, .., W-1, W][8]), and the x-shift kx - 1 of a 64-pixel M-tile is a start
// offset of kx pixels (16 bytes each) in the MMA descriptor.  An M-tile is 64 output pixels of one
// row (W >= 64), so the MMAs are M = 64: the 1-CTA M = 64 accumulator puts its rows 16q .. 16q+15 in
// TMEM lanes 32q .. 32q+15, and a second tile whose address starts at lane 16 takes lanes
// 32q+16 .. 32q+31 (the interleaved layout), so two tiles share one set of COUT columns and a
// 32-lane tcgen05.ld gives each warp 16 pixels of each.  The CTA's 256 pixels are 4 tiles in 2
// column sets.
__host__ __device__ constexpr int rows_plane(int W) {  // padded pixels per channel chunk, = 1 (mod 8)
    return (((256 / W + 2) * (W + 2) + 7) / 8) * 8 + 1;
}
__host__ __device__ constexpr size_t rows_smem_bytes(int cin, int cout, int W) {
    // at least 29 KB: at most 7 CTAs per SM, so that their TMEM (64 columns each) always fits
    const size_t b = size_t(cin / 8) * rows_plane(W) * 16 + size_t(9) * (cin / 8) * cout * 16 + 64;
    return b < 29 * 1024 ? 29 * 1024 : b;
}

template <int CIN, int COUT, int MODE>
__global__ void __launch_bounds__(NT) conv3x3_rows_kernel(ConvArgs a) {
    constexpr int CC = CIN / 8;
    extern __shared__ __align__(1024) unsigned char smem[];
    const int W = a.W, H = a.H;
    const int TR = 256 / W, W2 = W + 2, PS = rows_plane(W), TPR = W / 64;
    uint4* Xs = reinterpret_cast<uint4*>(smem);   // [CC][PS]: rows of W + 2 padded pixels
    uint4* Wt = Xs + size_t(CC) * PS;              // [9][CC][COUT]
    uint64_t* bar = reinterpret_cast<uint64_t*>(Wt + 9 * CC * COUT);
    uint32_t* tslot = reinterpret_cast<uint32_t*>(bar + 1);
    const int tid = threadIdx.x, warp = tid >> 5, lane = tid & 31;
    const int n = blockIdx.y, y0 = blockIdx.x * TR;
    constexpr uint32_t kCols = (2 * COUT) < 32 ? 32 : 2 * COUT;

    if (warp == 0) tc::tmem_alloc(tslot, kCols);
    if (tid == 0) {
        tc::mbar_init(bar, 1);
        tc::fence_mbar_init();
    }
    // stage rows y0-1 .. y0+TR (periodic in y) once, with the periodic x-neighbours at both ends, and
    // the weights: asynchronous 16-byte copies, all in flight together, then one wait
    for (int e = tid; e < (TR + 2) * W * CC; e += NT) {
        const int cc = e % CC, t = e / CC, x = t % W, r = t / W;
        const int y = (y0 - 1 + r + H) % H;
        const uint4* src = a.X + (size_t(n * H + y) * W + x) * CC + cc;
        uint4* row = Xs + size_t(cc) * PS + r * W2;
        tc::cp_async16(row + x + 1, src);
        if (x == W - 1) tc::cp_async16(row, src);
        if (x == 0) tc::cp_async16(row + W + 1, src);
    }
    for (int e = tid; e < 9 * CC * COUT; e += NT) tc::cp_async16(Wt + e, a.Wb + e);
    tc::cp_async_wait_all();
    tc::fence_proxy_async_smem();
    tc::fence_before_sync();
    __syncthreads();
    tc::fence_after_sync();
    const uint32_t tmem = *tslot;

    if (tid == 0) {
        constexpr uint32_t idesc = tc::idesc_bf16_f32(64, COUT);
        const uint32_t xb = tc::smem_addr(Xs), wb = tc::smem_addr(Wt);
        const uint32_t lbo_a = uint32_t(PS) * 16, lbo_b = COUT * 16;
        for (int j = 0; j < 4; ++j) {  // tile j: row j / TPR, pixels (j % TPR) * 64 ..
            const int r = j / TPR, x0 = (j % TPR) * 64;
            const uint32_t d = tmem + (uint32_t(16 * (j & 1)) << 16) + (j >> 1) * COUT;
            for (int sh = 0; sh < 9; ++sh) {
                const int ky = sh / 3, kx = sh % 3;
                for (int s = 0; s < CIN / 16; ++s) {
                    const uint32_t aa = xb + ((2 * s) * PS + (r + ky) * W2 + x0 + kx) * 16;
                    const uint32_t ba = wb + (sh * CC + 2 * s) * COUT * 16;
                    tc::mma_bf16(d, tc::smem_desc(aa, lbo_a, 128), tc::smem_desc(ba, lbo_b, 128), idesc, (sh | s) != 0);
                }
            }
        }
        tc::mma_commit(bar);
    }
    const bool ok = tc::mbar_wait_bounded(bar, 0, a.err);
    tc::fence_after_sync();
    if (ok) {
        for (int cs = 0; cs < 2; ++cs) {  // column set cs: tiles 2cs (lanes 0-15) and 2cs+1 (lanes 16-31)
            float acc[32];
            const uint32_t taddr = tmem + (uint32_t(warp * 32) << 16) + cs * COUT;
            if constexpr (COUT == 32) tc::tmem_ld_32x32(taddr, acc);
            else tc::tmem_ld_32x16(taddr, acc);
            const int j = 2 * cs + (lane >> 4);
            const int r = j / TPR, x = (j % TPR) * 64 + warp * 16 + (lane & 15);
            const size_t gp = size_t(n * H + y0 + r) * W + x;
            if constexpr (MODE == FVNET_CONV_HIDDEN) {
                float z[COUT], g[COUT];
#pragma unroll
                for (int c = 0; c < COUT; ++c) {
                    z[c] = acc[c] + a.bias[c];
                    g[c] = gelu_tanh(z[c]);
                }
                uint4* Zo = reinterpret_cast<uint4*>(a.Z + gp * COUT);
                uint4* Ao = reinterpret_cast<uint4*>(a.A + gp * COUT);
#pragma unroll
                for (int q = 0; q < COUT / 8; ++q) {
                    Zo[q] = pack8(z + 8 * q);
                    Ao[q] = pack8(g + 8 * q);
                }
            } else if constexpr (MODE == FVNET_CONV_OUTPUT) {
                float4 o = make_float4(acc[0] + a.bias[0], acc[1] + a.bias[1], acc[2] + a.bias[2], acc[3] + a.bias[3]);
                reinterpret_cast<float4*>(a.out4)[gp] = o;
            } else {
                float d[COUT];
                const uint4* Zp = reinterpret_cast<const uint4*>(a.Zprev + gp * COUT);
#pragma unroll
                for (int q = 0; q < COUT / 8; ++q) {
                    const uint4 u = Zp[q];
                    const __nv_bfloat16* zb = reinterpret_cast<const __nv_bfloat16*>(&u);
#pragma unroll
                    for (int jj = 0; jj < 8; ++jj) {
                        const float gz = (MODE == FVNET_CONV_BWD_GELU) ? gelu_tanh_grad(__bfloat162float(zb[jj])) : 1.0f;
                        d[8 * q + jj] = acc[8 * q + jj] * gz;
                    }
                }
                uint4* Ao = reinterpret_cast<uint4*>(a.A + gp * COUT);
#pragma unroll
                for (int q = 0; q < COUT / 8; ++q) Ao[q] = pack8(d + 8 * q);
            }
        }
    }
    tc::fence_before_sync();
    __syncthreads();
    if (warp == 0) tc::tmem_dealloc(tmem, kCols);
}

// ---- backward weights --------------------------------------------------------------------------
struct WgradArgs {
    const uint4* X;   // [B][H][W][CIN]
    const uint4* dZ;  // [B][H][W][COUT]
    float* partial;   // [gridDim.x][9*CIN][COUT]
    float* db_part;   // [gridDim.x][COUT]: the bias gradient of each CTA's rows
    int B, H, W;
    int rows_per_cta;
    int* err;
};

// ---- backward weights, operands read in place (MN-major) ----------------------------------------
// dW[(ky, kx, ci)][co] = sum over pixels of X[y + ky - 1][x + kx - 1][ci] dZ[y][x][co].  Per output row y
// and x-shift kx one accumulator D_kx[(ky, ci)][co] (M = 3 CIN rows, padded to 64 or 128; N = COUT; K =
// the row's pixels), and the MMAs read the staged rows themselves: a chunk of 8 channels is 16
// contiguous bytes per pixel and consecutive pixels are 16 bytes apart, which is the canonical
// no-swizzle MN-major layout (instruction descriptor major bits set; LBO = 128 bytes between groups
// of 8 pixels, SBO = the chunk stride).  There are no operand transposes.
// Input rows live in an 8-slot ring, each row stored twice (planes s and s + 8, s = (u + 1) mod 8 for
// image row u), so that the rows y - 1, y, y + 1 and one more are always 4 consecutive planes of CC
// chunks: the M rows (ky, ci) then have one chunk stride.  The fourth plane only feeds M rows past
// 3 CIN, whose results are not used.  An iteration takes two output rows of one image (one at an
// image's or range's end) with one MMA commit and one CTA barrier; while its MMAs run, the next
// iteration's new input rows are copied into slots that the MMAs read at most as an unused fourth
// plane, and its output-gradient rows into the other of two buffers.
__host__ __device__ constexpr size_t wgrad_mn_smem_bytes(int cin, int cout, int W) {
    // at least 46 KB: at most 4 CTAs per SM, so that their TMEM (up to 128 columns each) always fits
    const size_t b = size_t(16) * (cin / 8) * (W + 2) * 16 + size_t(4) * (cout / 8) * W * 16 + 64;
    return b < 46 * 1024 ? 46 * 1024 : b;
}

template <int CIN, int COUT>
__global__ void __launch_bounds__(NT) conv3x3_wgrad_mn_kernel(WgradArgs a) {
    constexpr int CC = CIN / 8, OC = COUT / 8, M9 = 9 * CIN;
    constexpr int MM = (3 * CIN) <= 64 ? 64 : 128;  // MMA M
    static_assert(3 * CIN <= 128, "three input rows of CIN channels fit one M = 128 accumulator");
    constexpr uint32_t kCols = (3 * COUT) <= 32 ? 32 : ((3 * COUT) <= 64 ? 64 : 128);
    extern __shared__ __align__(1024) unsigned char smem[];
    const int W = a.W, H = a.H, W2 = W + 2;
    uint4* Xs = reinterpret_cast<uint4*>(smem);    // [16 planes][CC][W + 2]: pixels x = -1 .. W
    uint4* Ds = Xs + size_t(16) * CC * W2;         // [2 buffers][2 rows][OC][W]
    uint64_t* bar = reinterpret_cast<uint64_t*>(Ds + size_t(4) * OC * W);
    uint32_t* tslot = reinterpret_cast<uint32_t*>(bar + 1);
    const int tid = threadIdx.x, warp = tid >> 5, lane = tid & 31;
    const int total = a.B * H;
    const int r0 = blockIdx.x * a.rows_per_cta, r1 = min(total, r0 + a.rows_per_cta);

    if (warp == 0) tc::tmem_alloc(tslot, kCols);
    if (tid == 0) {
        tc::mbar_init(bar, 1);
        tc::fence_mbar_init();
    }
    // input row u (image n, u in [-1, H], periodic) into its two planes, with the periodic x-neighbours
    auto stage_x = [&](int n, int u) {
        const int yr = (u + H) % H, s = (u + 1) & 7;
        const uint4* src = a.X + size_t(n * H + yr) * W * CC;
        for (int e = tid; e < W * CC; e += NT) {
            const int x = e / CC, cc = e - x * CC;
            for (int p = s; p < 16; p += 8) {
                uint4* row = Xs + (size_t(p) * CC + cc) * W2;
                tc::cp_async16(row + x + 1, src + e);
                if (x == W - 1) tc::cp_async16(row, src + e);
                if (x == 0) tc::cp_async16(row + W + 1, src + e);
            }
        }
    };
    auto stage_dz = [&](int n, int y, int buf, int j) {  // output-gradient row y into buffer buf, row j: [oc][x]
        const uint4* src = a.dZ + size_t(n * H + y) * W * OC;
        for (int e = tid; e < W * OC; e += NT) {
            const int x = e / OC, oc = e - x * OC;
            tc::cp_async16(Ds + ((size_t(buf) * 2 + j) * OC + oc) * W + x, src + e);
        }
    };
    // output rows an iteration starting at `row` takes: two of one image, one at an image's or range's end
    auto rows_in = [&](int row) { return (row + 1 < r1 && (row + 1) % H != 0) ? 2 : 1; };
    int cur = 0;
    if (r0 < r1) {
        const int n = r0 / H, y = r0 % H, k = rows_in(r0);
        for (int u = y - 1; u <= y + k; ++u) stage_x(n, u);
        for (int j = 0; j < k; ++j) stage_dz(n, y + j, 0, j);
    }
    tc::cp_async_wait_all();
    tc::fence_proxy_async_smem();
    tc::fence_before_sync();
    __syncthreads();
    tc::fence_after_sync();
    const uint32_t tmem = *tslot;
    constexpr uint32_t idesc = tc::idesc_bf16_f32(MM, COUT) | (1u << 15) | (1u << 16);  // A and B MN-major
    const uint32_t xb = tc::smem_addr(Xs), db = tc::smem_addr(Ds);
    const uint32_t sbo_a = uint32_t(W2) * 16, sbo_b = uint32_t(W) * 16;
    uint32_t phase = 0;
    bool ok = true;
    float bacc = 0.0f;
    for (int row = r0; row < r1;) {
        const int n = row / H, y = row % H, k = rows_in(row);
        if (tid == 0) {
            for (int j = 0; j < k; ++j) {
                const int p0 = (y + j) & 7;  // planes p0 .. p0 + 2 hold rows y + j - 1 .. y + j + 1
                for (int kx = 0; kx < 3; ++kx)
                    for (int ks = 0; ks < W / 16; ++ks) {
                        const uint32_t aa = xb + (uint32_t(p0 * CC) * W2 + 16 * ks + kx) * 16;
                        const uint32_t ba = db + (uint32_t((cur * 2 + j) * OC) * W + 16 * ks) * 16;
                        tc::mma_bf16(tmem + kx * COUT, tc::smem_desc(aa, 128, sbo_a), tc::smem_desc(ba, 128, sbo_b),
                                     idesc, (row > r0 || j > 0 || ks > 0) ? 1u : 0u);
                    }
            }
            tc::mma_commit(bar);
        }
        const int nrow = row + k;
        const bool has_next = nrow < r1, next_cont = has_next && (nrow % H) != 0;
        const int k2 = has_next ? rows_in(nrow) : 0;
        if (next_cont) {  // during the MMAs: the next iteration's new input rows and its dZ rows
            for (int u = y + k + 1; u <= y + k + k2; ++u) stage_x(n, u);
            for (int j = 0; j < k2; ++j) stage_dz(n, y + k + j, cur ^ 1, j);
        }
        {  // the bias gradient: thread t sums channel t % COUT over pixels t / COUT, + NT / COUT, .. of the rows
            const int co = tid % COUT;
            for (int j = 0; j < k; ++j) {
                const __nv_bfloat16* dz = reinterpret_cast<const __nv_bfloat16*>(Ds + size_t(cur * 2 + j) * OC * W);
                for (int x = tid / COUT; x < W; x += NT / COUT) bacc += __bfloat162float(dz[(size_t(co / 8) * W + x) * 8 + co % 8]);
            }
        }
        ok = tc::mbar_wait_bounded(bar, phase, a.err);
        phase ^= 1;
        tc::fence_after_sync();
        if (has_next && !next_cont) {  // a new image: its rows, now that the MMAs are done
            const int n2 = nrow / H;
            for (int u = -1; u <= k2; ++u) stage_x(n2, u);
            for (int j = 0; j < k2; ++j) stage_dz(n2, j, cur ^ 1, j);
        }
        tc::cp_async_wait_all();
        tc::fence_proxy_async_smem();
        tc::fence_before_sync();
        const int all_ok = __syncthreads_and(ok ? 1 : 0);  // the next iteration's data is visible
        tc::fence_after_sync();
        ok = all_ok != 0;
        if (!ok) break;  // a wait ran out (the error flag is set): the whole CTA leaves
        cur ^= 1;
        row = nrow;
    }
    if (ok && r0 < r1) {
        for (int kx = 0; kx < 3; ++kx) {
            float acc[32];
            const uint32_t taddr = tmem + (uint32_t(warp * 32) << 16) + kx * COUT;
            if constexpr (COUT == 32) tc::tmem_ld_32x32(taddr, acc);
            else tc::tmem_ld_32x16(taddr, acc);
            // M = 128: accumulator row m in lane m; M = 64: rows 16q .. 16q+15 in lanes 32q .. 32q+15
            const int mrow = (MM == 128) ? warp * 32 + lane : (lane < 16 ? warp * 16 + lane : 3 * CIN);
            if (mrow < 3 * CIN) {
                const int ky = mrow / CIN, ci = mrow - ky * CIN;
                const int m = (ky * 3 + kx) * CIN + ci;
                float* dst = a.partial + (size_t(blockIdx.x) * M9 + m) * COUT;
#pragma unroll
                for (int c = 0; c < COUT; ++c) dst[c] = acc[c];
            }
        }
    }
    __shared__ float sb[NT];
    sb[tid] = bacc;
    tc::fence_before_sync();
    __syncthreads();
    if (ok && r0 < r1 && tid < COUT) {  // the CTA's bias gradient, its threads' sums in a fixed order
        float b = 0.0f;
        for (int k = tid; k < NT; k += COUT) b += sb[k];
        a.db_part[size_t(blockIdx.x) * COUT + tid] = b;
    }
    if (warp == 0) tc::tmem_dealloc(tmem, kCols);
}

// dW[co][ci][ky][kx] = sum over CTAs (fixed order) of partial[cta][(ky*3+kx)*cin_pad + ci][co].  Thread
// f = (k*cin + ci)*cout + co: consecutive threads read consecutive co of a partial (coalesced).
__global__ void wgrad_reduce_kernel(const float* __restrict__ partial, int nparts, int cin_pad, int cout_pad,
                                    int cin, int cout, float* __restrict__ dW) {
    const int f = blockIdx.x * blockDim.x + threadIdx.x;
    if (f >= cout * cin * 9) return;
    const int co = f % cout, ci = (f / cout) % cin, k = f / (cout * cin);
    const size_t stride = size_t(9) * cin_pad * cout_pad;
    const size_t off = (size_t(k) * cin_pad + ci) * cout_pad + co;
    float s = 0.0f;
    for (int p = 0; p < nparts; ++p) s += partial[p * stride + off];
    dW[(size_t(co) * cin + ci) * 9 + k] = s;
}

// db[co] = sum over pixels of dZ[p][co]: the weight-gradient kernel leaves each CTA's sum over its rows
// in db_part[cta][co] (cout_pad per CTA); this sums them over the CTAs in a fixed order.
__global__ void bias_grad_reduce_kernel(const float* __restrict__ part, int nparts, int cout_pad, int cout,
                                        float* __restrict__ db) {
    const int co = threadIdx.x;
    if (co >= cout) return;
    float s = 0.0f;
    for (int p = 0; p < nparts; ++p) s += part[p * cout_pad + co];
    db[co] = s;
}

// Canonical fp32 weights W[co][ci][3][3] -> bf16 B-operand packs for the forward pass
// ([sh][cin_pad/8][cout_pad][8]) and the backward-data pass (transposed, spatially flipped:
// [sh'][cout_pad/8][cin_pad][8] with element W[co][ci][2-ky'][2-kx']).  Padding is zero.
__global__ void pack_weights_kernel(const float* __restrict__ Wc, int cout, int cin, int cout_pad, int cin_pad,
                                    __nv_bfloat16* __restrict__ Wf, __nv_bfloat16* __restrict__ Wbk) {
    const int nf = 9 * cin_pad * cout_pad;
    for (int e = blockIdx.x * blockDim.x + threadIdx.x; e < nf; e += gridDim.x * blockDim.x) {
        // forward: e = ((sh*CC + cc)*cout_pad + co)*8 + j, ci = cc*8 + j
        {
            const int j = e % 8, co = (e / 8) % cout_pad, cc = (e / (8 * cout_pad)) % (cin_pad / 8),
                      sh = e / (8 * cout_pad * (cin_pad / 8));
            const int ci = cc * 8 + j, ky = sh / 3, kx = sh % 3;
            const float w = (co < cout && ci < cin) ? Wc[((co * cin + ci) * 3 + ky) * 3 + kx] : 0.0f;
            Wf[e] = __float2bfloat16_rn(w);
        }
        // backward data: e = ((sh*CC' + cc)*cin_pad + ci)*8 + j, co = cc*8 + j, CC' = cout_pad/8
        {
            const int j = e % 8, ci = (e / 8) % cin_pad, cc = (e / (8 * cin_pad)) % (cout_pad / 8),
                      sh = e / (8 * cin_pad * (cout_pad / 8));
            const int co = cc * 8 + j, ky = 2 - sh / 3, kx = 2 - sh % 3;
            const float w = (co < cout && ci < cin) ? Wc[((co * cin + ci) * 3 + ky) * 3 + kx] : 0.0f;
            Wbk[e] = __float2bfloat16_rn(w);
        }
    }
}

template <int CIN, int COUT, int MODE>
int launch_conv(const ConvArgs& a, cudaStream_t st) {
    if (a.W >= 64 && getenv("FVNET_CONV_COPIES") == nullptr) {  // one staged copy (FVNET_CONV_COPIES: three)
        static bool rattr = false;
        if (!rattr) {  // the limit for the largest image width served (W = 256)
            if (cudaFuncSetAttribute(conv3x3_rows_kernel<CIN, COUT, MODE>, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                     (int)rows_smem_bytes(CIN, COUT, 256)) != cudaSuccess)
                return fv_internal_set_error(FVNET_ERR_CUDA, "fvnet: smem attribute");
            rattr = true;
        }
        conv3x3_rows_kernel<CIN, COUT, MODE><<<dim3(a.H / (256 / a.W), a.B), NT, rows_smem_bytes(CIN, COUT, a.W), st>>>(a);
        return FVNET_OK;
    }
    const size_t smem = conv_smem_bytes(CIN, COUT, a.W);
    static bool attr = false;
    if (!attr) {  // the limit for the largest image width served (W = 256)
        if (cudaFuncSetAttribute(conv3x3_kernel<CIN, COUT, MODE>, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                 (int)conv_smem_bytes(CIN, COUT, 256)) != cudaSuccess)
            return fv_internal_set_error(FVNET_ERR_CUDA, "fvnet: smem attribute");
        attr = true;
    }
    dim3 grid(a.H / (256 / a.W), a.B);
    conv3x3_kernel<CIN, COUT, MODE><<<grid, NT, smem, st>>>(a);
    return FVNET_OK;
}

template <int CIN, int COUT>
int launch_wgrad(const WgradArgs& a, int nparts, cudaStream_t st) {
    static bool attr = false;
    if (!attr) {  // the limit for the largest image width served (W = 128)
        if (cudaFuncSetAttribute(conv3x3_wgrad_mn_kernel<CIN, COUT>, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                 (int)wgrad_mn_smem_bytes(CIN, COUT, 128)) != cudaSuccess)
            return fv_internal_set_error(FVNET_ERR_CUDA, "fvnet: smem attribute");
        attr = true;
    }
    conv3x3_wgrad_mn_kernel<CIN, COUT><<<nparts, NT, wgrad_mn_smem_bytes(CIN, COUT, a.W), st>>>(a);
    return FVNET_OK;
}

bool shape_ok(int B, int H, int W) {
    return B > 0 && (W == 32 || W == 64 || W == 128 || W == 256) && H > 0 && H % (256 / W) == 0;
}

}  // namespace fvnet

using namespace fvnet;

extern "C" {

int fvnet_conv3x3(int mode, int cin_pad, int cout_pad, int B, int H, int W, const void* X, const void* Wpacked,
                  const float* bias, const void* Zprev, void* Z, void* A, float* out4, int* err, void* stream) {
    if (!shape_ok(B, H, W) || !X || !Wpacked) return fv_internal_set_error(FVNET_ERR_ARG, "fvnet_conv3x3: bad shape or NULL input");
    ConvArgs a{};
    a.X = static_cast<const uint4*>(X);
    a.Wb = static_cast<const uint4*>(Wpacked);
    a.bias = bias;
    a.Zprev = static_cast<const __nv_bfloat16*>(Zprev);
    a.Z = static_cast<__nv_bfloat16*>(Z);
    a.A = static_cast<__nv_bfloat16*>(A);
    a.out4 = out4;
    a.B = B; a.H = H; a.W = W; a.err = err;
    cudaStream_t st = static_cast<cudaStream_t>(stream);
    int rc = FVNET_ERR_ARG;
    if (mode == FVNET_CONV_HIDDEN) {
        if (!bias || !Z || !A) return fv_internal_set_error(FVNET_ERR_ARG, "fvnet_conv3x3: hidden needs bias, Z, A");
        if (cin_pad == 16 && cout_pad == 32) rc = launch_conv<16, 32, FVNET_CONV_HIDDEN>(a, st);
        else if (cin_pad == 32 && cout_pad == 32) rc = launch_conv<32, 32, FVNET_CONV_HIDDEN>(a, st);
    } else if (mode == FVNET_CONV_OUTPUT) {
        if (!bias || !out4) return fv_internal_set_error(FVNET_ERR_ARG, "fvnet_conv3x3: output needs bias, out4");
        if (cin_pad == 32 && cout_pad == 16) rc = launch_conv<32, 16, FVNET_CONV_OUTPUT>(a, st);
    } else if (mode == FVNET_CONV_BWD_GELU) {
        if (!Zprev || !A) return fv_internal_set_error(FVNET_ERR_ARG, "fvnet_conv3x3: backward needs Zprev, A");
        if (cin_pad == 16 && cout_pad == 32) rc = launch_conv<16, 32, FVNET_CONV_BWD_GELU>(a, st);
        else if (cin_pad == 32 && cout_pad == 32) rc = launch_conv<32, 32, FVNET_CONV_BWD_GELU>(a, st);
    } else if (mode == FVNET_CONV_BWD_PLAIN) {
        if (!A) return fv_internal_set_error(FVNET_ERR_ARG, "fvnet_conv3x3: backward needs A");
        if (cin_pad == 16 && cout_pad == 32) rc = launch_conv<16, 32, FVNET_CONV_BWD_PLAIN>(a, st);
        else if (cin_pad == 32 && cout_pad == 32) rc = launch_conv<32, 32, FVNET_CONV_BWD_PLAIN>(a, st);
        else if (cin_pad == 32 && cout_pad == 16) rc = launch_conv<32, 16, FVNET_CONV_BWD_PLAIN>(a, st);
    }
    if (rc == FVNET_ERR_ARG) return fv_internal_set_error(FVNET_ERR_ARG, "fvnet_conv3x3: unsupported mode/channels");
    if (rc) return rc;
    const cudaError_t e = cudaGetLastError();
    if (e != cudaSuccess) return fv_internal_set_error(FVNET_ERR_CUDA, cudaGetErrorString(e));
    return FVNET_OK;
}

// 2 CTAs per SM (296 partial sums): 3 or 4 per SM were slower (more partial sums to reduce), 1 per SM
// within 1 %
int fvnet_wgrad_parts(int B, int H) { return std::max(1, std::min(2 * 148, B * H)); }

int fvnet_conv3x3_wgrad(int cin_pad, int cout_pad, int cin, int cout, int B, int H, int W, const void* X, const void* dZ,
                        float* partial, float* dW, float* db, float* db_part, int* err, void* stream) {
    if (!shape_ok(B, H, W) || W > 128 || !X || !dZ || !partial || !dW || !db || !db_part || cin > cin_pad ||
        cout > cout_pad)
        return fv_internal_set_error(FVNET_ERR_ARG, "fvnet_conv3x3_wgrad: bad arguments");
    cudaStream_t st = static_cast<cudaStream_t>(stream);
    const int nparts = fvnet_wgrad_parts(B, H);
    WgradArgs a{};
    a.X = static_cast<const uint4*>(X);
    a.dZ = static_cast<const uint4*>(dZ);
    a.partial = partial;
    a.db_part = db_part;
    a.B = B; a.H = H; a.W = W;
    a.rows_per_cta = (B * H + nparts - 1) / nparts;
    a.err = err;
    int rc = FVNET_ERR_ARG;
    if (cin_pad == 16 && cout_pad == 32) rc = launch_wgrad<16, 32>(a, nparts, st);
    else if (cin_pad == 32 && cout_pad == 32) rc = launch_wgrad<32, 32>(a, nparts, st);
    else if (cin_pad == 32 && cout_pad == 16) rc = launch_wgrad<32, 16>(a, nparts, st);
    if (rc == FVNET_ERR_ARG) return fv_internal_set_error(FVNET_ERR_ARG, "fvnet_conv3x3_wgrad: unsupported channels");
    if (rc) return rc;
    // parts actually used: CTAs whose row range is not empty
    const int used = (B * H + a.rows_per_cta - 1) / a.rows_per_cta;
    wgrad_reduce_kernel<<<(cout * cin * 9 + 255) / 256, 256, 0, st>>>(partial, used, cin_pad, cout_pad, cin, cout, dW);
    bias_grad_reduce_kernel<<<1, 64, 0, st>>>(db_part, used, cout_pad, cout, db);
    const cudaError_t e = cudaGetLastError();
    if (e != cudaSuccess) return fv_internal_set_error(FVNET_ERR_CUDA, cudaGetErrorString(e));
    return FVNET_OK;
}

int fvnet_pack_weights(int cout, int cin, int cout_pad, int cin_pad, const float* W, void* Wfwd, void* Wbwd,
                       void* stream) {
    if (!W || !Wfwd || !Wbwd || cout > cout_pad || cin > cin_pad || cin_pad % 8 || cout_pad % 8)
        return fv_internal_set_error(FVNET_ERR_ARG, "fvnet_pack_weights: bad arguments");
    const int nf = 9 * cin_pad * cout_pad;
    pack_weights_kernel<<<(nf + 255) / 256, 256, 0, static_cast<cudaStream_t>(stream)>>>(
        W, cout, cin, cout_pad, cin_pad, static_cast<__nv_bfloat16*>(Wfwd), static_cast<__nv_bfloat16*>(Wbwd));
    const cudaError_t e = cudaGetLastError();
    if (e != cudaSuccess) return fv_internal_set_error(FVNET_ERR_CUDA, cudaGetErrorString(e));
    return FVNET_OK;
}

}  // extern "C"
