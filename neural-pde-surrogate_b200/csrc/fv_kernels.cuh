// Kernels of the finite-volume step (one fused kernel per SSP-RK2 stage), the on-device time
// control, the wave-speed / positivity reduction and the trajectory block average.
//
// Stage kernel (one CTA per TX x TY tile of interior cells, NT threads):
//   P1  load the tile plus a 2-cell halo of the stage input (ghosts resolved by bc_index: periodic
//       wrap or transmissive clamp, grid2d.hpp:43-66), convert to primitives      -> smem W
//   P2  limited slopes in x (cells -1..TX) and y (rows -1..TY)  (solver2d.hpp:142-143,159-162)
//   P3  x-face fluxes F (TX+1 per row) and y-face fluxes G (TY+1 per column), the y-faces through
//       the momentum swap (riemann2d.hpp:42-44)                                    -> smem F, G
//   P4  L = -(F_r - F_l)/dx - (G_t - G_b)/dy in the reference's accumulation order
//       (solver2d.hpp:141,149-150,176-177), then the stage update (solver2d.hpp:92 / :100).
//       Stage 2 also reduces the next step's CFL wave speeds and the first non-physical cell
//       (compute_dt, solver2d.hpp:67-83) into the control block: dt never leaves the device.
#pragma once
#include <climits>
#include "fv_physics.cuh"

namespace fv {

constexpr int TX = 32, TY = 16, NT = 256;
constexpr int HX = TX + 4, HY = TY + 4;  // loaded tile with its 2-cell halo
constexpr int SXW = TX + 2;              // x-slopes per row: cells -1..TX
constexpr int SYH = TY + 2;              // y-slope rows: -1..TY
constexpr int FXW = TX + 1;              // x-faces per row
constexpr int GYH = TY + 1;              // y-face rows
constexpr int NFX = TY * FXW, NFY = GYH * TX;

struct StageSmem {
    Q4 W[HY][HX];
    Q4 dWx[TY][SXW];
    Q4 dWy[SYH][TX];
    Q4 F[TY][FXW];
    Q4 G[GYH][TX];
};

enum : int { MODE_LOOP = 0, MODE_FIXED = 1 };

// Control block of one grid (device memory).  Fields are double-buffered by step parity so that a
// kernel never reads a field another CTA of the same kernel writes:
//   stage 1 reads step, t[par], sxy[par], bad[par] and (CTA 0 only) writes dt, t[par^1], par2, run2
//   and resets sxy[par^1], bad[par^1]; stage 2 reads dt, par2, run2, accumulates into sxy[par2],
//   bad[par2] and (CTA 0 only) increments step.
struct FvCtrl {
    unsigned long long sxy[2][2];  // bit patterns of the non-negative max wave speeds (x, y)
    int bad[2];                    // min row-major index of a non-physical cell, INT_MAX if none
    int par2, run2;
    double t[2];
    double dt;                     // dt of the step in flight
    double t_next;                 // target of fv_advance_to
    double dt_fixed;               // dt of fv_step
    long long step;                // steps taken
    int mode;
    int status;                    // 0, or FV_ERR_NONPHYSICAL
    int bad_index;                 // row-major index recorded with status
    int pad_;
};

struct StageArgs {
    const Q4* Uin;    // state whose RHS is evaluated: U (stage 1) or U1 (stage 2)
    const Q4* Ubase;  // U (stage 2)
    Q4* Uout;         // U1 (stage 1) or U in place (stage 2)
    int nx, ny, bc_x, bc_y;
    double cx, cy;    // 1.0/dx and 1.0/dy, as the reference writes (1.0 / g.dx)
    double dx, dy, cfl;
    FvCtrl* ctrl;
};

__device__ __forceinline__ double warp_max(double v) {
#pragma unroll
    for (int o = 16; o > 0; o >>= 1) v = smax(v, __shfl_xor_sync(0xffffffffu, v, o));
    return v;
}
__device__ __forceinline__ int warp_min_int(int v) {
#pragma unroll
    for (int o = 16; o > 0; o >>= 1) v = min(v, __shfl_xor_sync(0xffffffffu, v, o));
    return v;
}

// compute_dt's per-cell work (solver2d.hpp:74-78): non-physical cells are recorded, not maxed.
__device__ __forceinline__ void wave_speed_cell(const Q4& U, int lin, double& sx, double& sy, int& bad) {
    Q4 W = to_primitive(U);
    if (!(W.a > 0.0) || !(W.d > 0.0)) {
        bad = min(bad, lin);
        return;
    }
    double a = sound_speed(W);
    sx = smax(sx, fabs(W.b) + a);
    sy = smax(sy, fabs(W.c) + a);
}

// Block-wide reduction of (sx, sy, bad) into ctrl slot `par` (atomics; max/min are order-free, so
// the result is deterministic).  Must be called by all NT threads.
__device__ __forceinline__ void reduce_wave_speeds(double sx, double sy, int bad, FvCtrl* c, int par) {
    __shared__ double rsx[NT / 32], rsy[NT / 32];
    __shared__ int rbad[NT / 32];
    sx = warp_max(sx);
    sy = warp_max(sy);
    bad = warp_min_int(bad);
    const int w = threadIdx.x >> 5, l = threadIdx.x & 31;
    if (l == 0) { rsx[w] = sx; rsy[w] = sy; rbad[w] = bad; }
    __syncthreads();
    if (w == 0) {
        sx = l < NT / 32 ? rsx[l] : 0.0;
        sy = l < NT / 32 ? rsy[l] : 0.0;
        bad = l < NT / 32 ? rbad[l] : INT_MAX;
        sx = warp_max(sx);
        sy = warp_max(sy);
        bad = warp_min_int(bad);
        if (l == 0) {
            if (sx > 0.0) atomicMax(&c->sxy[par][0], (unsigned long long)__double_as_longlong(sx));
            if (sy > 0.0) atomicMax(&c->sxy[par][1], (unsigned long long)__double_as_longlong(sy));
            if (bad != INT_MAX) atomicMin(&c->bad[par], bad);
        }
    }
}

template <int FLUX, int LIM, int STAGE>
__global__ void __launch_bounds__(NT, 2) stage_kernel(StageArgs a) {
    extern __shared__ __align__(16) unsigned char smem_raw[];
    StageSmem& s = *reinterpret_cast<StageSmem*>(smem_raw);
    FvCtrl* c = a.ctrl;
    const bool cta0 = (blockIdx.x == 0 && blockIdx.y == 0);
    double dt;
    int par2 = 0;

    if constexpr (STAGE == 1) {
        // ---- step control: dt = min(compute_dt(U), t_next - t) (main2d.cpp:238, solver2d.hpp:82) ----
        const long long step = c->step;
        const int par = int(step & 1);
        const double t = c->t[par];
        bool active = true;
        if (c->mode == MODE_FIXED) {
            dt = c->dt_fixed;
        } else {
            active = (c->status == 0) && (t < c->t_next);
            if (active && c->bad[par] != INT_MAX) {
                active = false;
                if (cta0 && threadIdx.x == 0) {
                    c->status = 3;  // FV_ERR_NONPHYSICAL
                    c->bad_index = c->bad[par];
                }
            }
            dt = 0.0;
            if (active) {
                const double sx = __longlong_as_double((long long)c->sxy[par][0]);
                const double sy = __longlong_as_double((long long)c->sxy[par][1]);
                dt = smin(a.cfl / (sx / a.dx + sy / a.dy), c->t_next - t);
            }
        }
        if (cta0 && threadIdx.x == 0) {
            c->run2 = active ? 1 : 0;
            if (active) {
                c->dt = dt;
                // fv_step mirrors Solver::step, which has no notion of time: only the loop advances t
                c->t[par ^ 1] = (c->mode == MODE_FIXED) ? t : t + dt;
                c->par2 = par ^ 1;
                c->sxy[par ^ 1][0] = 0ull;
                c->sxy[par ^ 1][1] = 0ull;
                c->bad[par ^ 1] = INT_MAX;
            }
        }
        if (!active) return;
    } else {
        if (!c->run2) return;
        dt = c->dt;
        par2 = c->par2;
    }

    const int nx = a.nx, ny = a.ny;
    const int i0 = blockIdx.x * TX, j0 = blockIdx.y * TY;
    const Q4* __restrict__ Uin = a.Uin;

    // P1: halo tile -> primitives (solver2d.hpp:133-134 on the ghost-filled array)
    for (int e = threadIdx.x; e < HX * HY; e += NT) {
        const int r = e / HX, col = e - r * HX;
        const int gi = bc_index(i0 - 2 + col, nx, a.bc_x);
        const int gj = bc_index(j0 - 2 + r, ny, a.bc_y);
        st_q4(&s.W[r][col], to_primitive(ldg_q4(Uin + (size_t)gj * nx + gi)));
    }
    __syncthreads();

    // P2: limited slopes
    for (int e = threadIdx.x; e < TY * SXW + SYH * TX; e += NT) {
        if (e < TY * SXW) {
            const int r = e / SXW, k = e - r * SXW;  // cell (k-1, r): W[r+2][k+1]
            st_q4(&s.dWx[r][k], limited_slope<LIM>(ld_q4(&s.W[r + 2][k]), ld_q4(&s.W[r + 2][k + 1]),
                                                   ld_q4(&s.W[r + 2][k + 2])));
        } else {
            const int e2 = e - TY * SXW;
            const int r = e2 / TX, k = e2 - r * TX;  // cell (k, r-1): W[r+1][k+2]
            st_q4(&s.dWy[r][k], limited_slope<LIM>(ld_q4(&s.W[r][k + 2]), ld_q4(&s.W[r + 1][k + 2]),
                                                   ld_q4(&s.W[r + 2][k + 2])));
        }
    }
    __syncthreads();

    // P3: face fluxes, flux(to_conserved(edge(W_L, dW_L, +1)), to_conserved(edge(W_R, dW_R, -1)))
    for (int e = threadIdx.x; e < NFX + NFY; e += NT) {
        const Q4 *wl, *dl, *wr, *dr;
        Q4* out;
        bool ydir;
        if (e < NFX) {  // x-face f of row r, between cells f-1 and f (solver2d.hpp:145-148)
            const int r = e / FXW, f = e - r * FXW;
            wl = &s.W[r + 2][f + 1]; dl = &s.dWx[r][f];
            wr = &s.W[r + 2][f + 2]; dr = &s.dWx[r][f + 1];
            out = &s.F[r][f];
            ydir = false;
        } else {        // y-face g of column k, between rows g-1 and g (solver2d.hpp:165-169)
            const int e2 = e - NFX;
            const int g = e2 / TX, k = e2 - g * TX;
            wl = &s.W[g + 1][k + 2]; dl = &s.dWy[g][k];
            wr = &s.W[g + 2][k + 2]; dr = &s.dWy[g + 1][k];
            out = &s.G[g][k];
            ydir = true;
        }
        Q4 UL = to_conserved(edge(ld_q4(wl), ld_q4(dl), +1.0));
        Q4 UR = to_conserved(edge(ld_q4(wr), ld_q4(dr), -1.0));
        if (ydir) { UL = swap_xy(UL); UR = swap_xy(UR); }
        Q4 F = face_flux<FLUX>(UL, UR);
        if (ydir) F = swap_xy(F);
        st_q4(out, F);
    }
    __syncthreads();

    // P4: divergence + stage update
    double sx = 0.0, sy = 0.0;
    int bad = INT_MAX;
    const double cx = a.cx, cy = a.cy;
    for (int e = threadIdx.x; e < TX * TY; e += NT) {
        const int r = e / TX, k = e - r * TX;
        const int i = i0 + k, j = j0 + r;
        if (i >= nx || j >= ny) continue;
        const Q4 Fl = ld_q4(&s.F[r][k]), Fr = ld_q4(&s.F[r][k + 1]);
        const Q4 Gb = ld_q4(&s.G[r][k]), Gt = ld_q4(&s.G[r + 1][k]);
        Q4 L;
        L.a = (0.0 + cx * Fl.a) - cx * Fr.a;
        L.b = (0.0 + cx * Fl.b) - cx * Fr.b;
        L.c = (0.0 + cx * Fl.c) - cx * Fr.c;
        L.d = (0.0 + cx * Fl.d) - cx * Fr.d;
        L.a = L.a + cy * Gb.a; L.a = L.a - cy * Gt.a;
        L.b = L.b + cy * Gb.b; L.b = L.b - cy * Gt.b;
        L.c = L.c + cy * Gb.c; L.c = L.c - cy * Gt.c;
        L.d = L.d + cy * Gb.d; L.d = L.d - cy * Gt.d;
        const size_t idx = (size_t)j * nx + i;
        if constexpr (STAGE == 1) {
            const Q4 u = ldg_q4(Uin + idx);
            st_q4(a.Uout + idx, Q4{u.a + dt * L.a, u.b + dt * L.b, u.c + dt * L.c, u.d + dt * L.d});
        } else {
            const Q4 u = ld_q4(a.Ubase + idx);
            const Q4 u1 = ldg_q4(Uin + idx);
            const Q4 un{0.5 * (u.a + u1.a + dt * L.a), 0.5 * (u.b + u1.b + dt * L.b),
                        0.5 * (u.c + u1.c + dt * L.c), 0.5 * (u.d + u1.d + dt * L.d)};
            st_q4(a.Uout + idx, un);
            wave_speed_cell(un, (int)idx, sx, sy, bad);
        }
    }
    if constexpr (STAGE == 2) {
        reduce_wave_speeds(sx, sy, bad, c, par2);
        if (cta0 && threadIdx.x == 0) c->step = c->step + 1;
    }
}

// Wave speeds / positivity of the current state into slot step&1 (after fv_set_state).
__global__ void __launch_bounds__(NT) wave_speed_kernel(const Q4* __restrict__ U, int n, FvCtrl* c) {
    const int par = int(c->step & 1);
    double sx = 0.0, sy = 0.0;
    int bad = INT_MAX;
    for (int k = blockIdx.x * NT + threadIdx.x; k < n; k += gridDim.x * NT)
        wave_speed_cell(ldg_q4(U + k), k, sx, sy, bad);
    reduce_wave_speeds(sx, sy, bad, c, par);
}

__global__ void ctrl_reset_kernel(FvCtrl* c, double t, int reset_step) {
    if (reset_step) c->step = 0;
    const int par = int(c->step & 1);
    c->sxy[par][0] = 0ull;
    c->sxy[par][1] = 0ull;
    c->bad[par] = INT_MAX;
    c->t[par] = t;
    c->status = 0;
    c->bad_index = -1;
    c->run2 = 0;
}

__global__ void ctrl_set_kernel(FvCtrl* c, int mode, double t_next, double dt_fixed) {
    c->mode = mode;
    c->t_next = t_next;
    c->dt_fixed = dt_fixed;
    if (mode == MODE_LOOP) c->status = 0;
}

__global__ void ctrl_set_time_kernel(FvCtrl* c, double t) { c->t[int(c->step & 1)] = t; }

// to_conserved of primitive fields (io_hdf5.hpp:197-204); counts cells with !(rho>0)||!(p>0).
__global__ void primitive_to_state_kernel(const double* __restrict__ rho, const double* __restrict__ u,
                                          const double* __restrict__ v, const double* __restrict__ p, int n,
                                          Q4* __restrict__ U, int* nbad) {
    for (int k = blockIdx.x * blockDim.x + threadIdx.x; k < n; k += gridDim.x * blockDim.x) {
        const Q4 W{rho[k], u[k], v[k], p[k]};
        if (!(W.a > 0.0) || !(W.d > 0.0)) atomicAdd(nbad, 1);
        st_q4(U + k, to_conserved(W));
    }
}

// TrajectoryWriter::add for one level (trajectory.hpp:31-51): one thread per coarse cell, the f x f
// sum in j-outer / i-inner order, times inv = 1.0/(double(f)*f), cast to float.
__global__ void block_average_kernel(const Q4* __restrict__ U, int nx, int ny, int f, double inv,
                                     float* __restrict__ out) {
    const int nxc = nx / f, nyc = ny / f;
    const int n = nxc * nyc;
    for (int e = blockIdx.x * blockDim.x + threadIdx.x; e < n; e += gridDim.x * blockDim.x) {
        const int jc = e / nxc, ic = e - jc * nxc;
        double s0 = 0.0, s1 = 0.0, s2 = 0.0, s3 = 0.0;
        for (int j = jc * f; j < (jc + 1) * f; ++j)
            for (int i = ic * f; i < (ic + 1) * f; ++i) {
                const Q4 q = ldg_q4(U + (size_t)j * nx + i);
                s0 += q.a; s1 += q.b; s2 += q.c; s3 += q.d;
            }
        const size_t plane = (size_t)nyc * nxc;
        out[e] = (float)(s0 * inv);
        out[plane + e] = (float)(s1 * inv);
        out[2 * plane + e] = (float)(s2 * inv);
        out[3 * plane + e] = (float)(s3 * inv);
    }
}

template <int FLUX>
__global__ void riemann_flux_kernel(int n, int y_face, const Q4* __restrict__ UL, const Q4* __restrict__ UR,
                                    Q4* __restrict__ F) {
    for (int k = blockIdx.x * blockDim.x + threadIdx.x; k < n; k += gridDim.x * blockDim.x) {
        Q4 l = ldg_q4(UL + k), r = ldg_q4(UR + k);
        if (y_face) { l = swap_xy(l); r = swap_xy(r); }
        Q4 f = face_flux<FLUX>(l, r);
        if (y_face) f = swap_xy(f);
        st_q4(F + k, f);
    }
}

// Ghosted copy of an interior state: cell (i, j) of the ring holds U[bc_index(i), bc_index(j)].
__global__ void fill_ghosts_kernel(int nx, int ny, int bc_x, int bc_y, const Q4* __restrict__ U, Q4* __restrict__ Ug) {
    const int W = nx + 4, n = W * (ny + 4);
    for (int k = blockIdx.x * blockDim.x + threadIdx.x; k < n; k += gridDim.x * blockDim.x) {
        const int j = k / W - 2, i = k % W - 2;
        st_q4(Ug + k, ldg_q4(U + (size_t)bc_index(j, ny, bc_y) * nx + bc_index(i, nx, bc_x)));
    }
}

}  // namespace fv
