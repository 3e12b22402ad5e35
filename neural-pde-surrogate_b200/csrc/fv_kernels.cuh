// Kernels of the finite-volume step (one fused kernel per SSP-RK2 stage), the on-device time
// control, the wave-speed / positivity reduction and the trajectory block average.
//
// Stage kernel, one CTA per TX x TY tile of interior cells (NT threads, one per cell):
//   P1  load the tile plus a 2-cell halo of the stage input (ghosts resolved by bc_index: periodic
//       wrap or transmissive clamp, grid2d.hpp:43-66), convert to primitives      -> smem W
//   P2  limited slopes in x (cells -1..TX) and y (rows -1..TY)  (solver2d.hpp:142-143,159-162)
//   P3  x-face fluxes F (TX+1 per row) and y-face fluxes G (TY+1 per column), the y-faces through
//       the momentum swap (riemann2d.hpp:42-44)                                    -> smem F, G
//   P4  L = -(F_r - F_l)/dx - (G_t - G_b)/dy in the reference's accumulation order
//       (solver2d.hpp:141,149-150,176-177), then the stage update (solver2d.hpp:92 / :100).
//       Stage 2 also reduces the next step's CFL wave speeds and the first non-physical cell
//       (compute_dt, solver2d.hpp:67-83) into the control block: dt never leaves the device.
// The primitive arrays W, W1 are stored in HBM as two planes of double2, (rho, u) and (v, p), the
// layout of the shared-memory tile: an interior tile's halo block is one TMA box (P1), boundary tiles
// load cell by cell through the BC index map.
// Every face flux is computed from the same inputs in the same order whatever the tile shape, so all
// tile shapes give bit-identical results; the shape is a tuning choice (fv_autotune).
#pragma once
#include <cuda.h>  // CUtensorMap

#include <climits>

#include "fv_physics.cuh"
#include "tc_sm100.cuh"

// Phase marker inside tile_body (no-op unless a build defines it, e.g. to record clock64()).
#ifndef FV_PHASE_MARK
#define FV_PHASE_MARK(k)
#endif

namespace fv {

// Shared-memory tile: every 4-vector field is two planes of double2, (q0, q1) and (q2, q3), so a Q4
// moves with two 16-byte accesses and consecutive cells of a warp hit consecutive 16-byte words
// (conflict-free).
template <int TX_, int TY_>
struct TileSmem {
    static constexpr int TX = TX_, TY = TY_, HX = TX + 4, HY = TY + 4;
    double2 W[2][HY][HX];        // primitives of the tile + 2-cell halo
    double2 dX[2][TY][TX + 2];   // x-slopes of cells -1..TX
    double2 dY[2][TY + 2][TX];   // y-slopes of rows -1..TY
    double2 F[2][TY][TX + 1];    // x-face fluxes
    double2 G[2][TY + 1][TX];    // y-face fluxes
    uint64_t bar;                // mbarrier of the P1 TMA load
};

template <int R, int Cc>
__device__ __forceinline__ Q4 lds(const double2 (&a)[2][R][Cc], int r, int c) {
    const double2 lo = a[0][r][c], hi = a[1][r][c];
    return Q4{lo.x, lo.y, hi.x, hi.y};
}
template <int R, int Cc>
__device__ __forceinline__ void sts(double2 (&a)[2][R][Cc], int r, int c, const Q4& q) {
    a[0][r][c] = make_double2(q.a, q.b);
    a[1][r][c] = make_double2(q.c, q.d);
}

enum : int { MODE_LOOP = 0, MODE_FIXED = 1 };

// Control block of one grid (device memory).  Fields are double-buffered by step parity so that a
// kernel never reads a field another CTA of the same kernel writes:
//   stage 1 reads step, t[par], sxy[par], bad[par] and (leader CTA only) writes dt, t[par^1],
//   par2, run2 and resets sxy[par^1], bad[par^1]; stage 2 reads dt, par2, run2, accumulates into
//   sxy[par2], bad[par2] and (leader only) increments step.
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
    int status;                    // 0, FV_ERR_NONPHYSICAL, or FV_ERR_TIMEOUT (a bounded wait ran out)
    int bad_index;                 // row-major index recorded with status
    int pad_;
    // persistent stepper (fv_stepper.cuh), one launch at a time: its work queue, and what each
    // completed step publishes for the next (step s's dt in sdt[s & 1], whether it runs in srun[s & 1])
    unsigned long long queue;      // next work item of the launch
    unsigned long long done2;      // stage-2 items completed in the launch
    long long complete;            // last step whose stage 2 has finished on every tile
    long long stop;                // first step that does not run (LLONG_MAX while unknown)
    long long s0, s_end;           // first step of the launch; steps < s_end may run
    double sdt[2];
    int srun[2];
};

// One grid as the stage kernels see it.  W and W1 hold to_primitive(U) and to_primitive(U1): each
// stage writes the primitives of the state it produces (it needs them anyway for the wave speeds or
// costs one conversion per cell), so the next stage loads its tile + halo as primitives instead of
// converting 1.4-1.7 cells per cell.  The conversion is deterministic, so the bits are unchanged.
struct GridDesc {
    Q4* U;            // state (stage 2 writes it in place)
    Q4* U1;           // intermediate RK stage
    Q4* W;            // to_primitive(U)
    Q4* W1;           // to_primitive(U1)
    int nx, ny, bc_x, bc_y;
    double dx, dy, cfl;
    double cx, cy;    // 1.0/dx and 1.0/dy, as the reference writes (1.0 / g.dx)
    FvCtrl* ctrl;
};

// TMA descriptors of one grid's W and W1 for one tile shape: 4-D (2 doubles, nx, ny, 2 planes) with
// box (2, TX + 4, TY + 4, 2) -- a tile's halo block of both planes.  Passed to the single-grid stage
// kernel as a __grid_constant__ parameter (a TMA descriptor must live in parameter, constant or
// global memory).
struct TileMaps {
    CUtensorMap w, w1;
    int use;  // 0: every tile loads through the BC index map
};

// Primitive arrays: plane 0 = (rho, u), plane 1 = (v, p), each n = nx * ny cells of double2.
__device__ __forceinline__ Q4 ldg_w(const Q4* W, size_t n, size_t k) {
    const double2* p = reinterpret_cast<const double2*>(W);
    const double2 lo = __ldg(p + k), hi = __ldg(p + n + k);
    return Q4{lo.x, lo.y, hi.x, hi.y};
}
// The same loads through L2 only (ld.global.cg), for data that other CTAs of the same launch wrote:
// the persistent stepper reads fields its own launch produced, which a non-coherent (__ldg) or
// L1-cached load could see stale.
__device__ __forceinline__ Q4 ldcg_w(const Q4* W, size_t n, size_t k) {
    const double2* p = reinterpret_cast<const double2*>(W);
    const double2 lo = __ldcg(p + k), hi = __ldcg(p + n + k);
    return Q4{lo.x, lo.y, hi.x, hi.y};
}
__device__ __forceinline__ Q4 ldcg_q4(const Q4* p) {
    const double2* v = reinterpret_cast<const double2*>(p);
    const double2 x = __ldcg(v), y = __ldcg(v + 1);
    return Q4{x.x, x.y, y.x, y.y};
}
__device__ __forceinline__ void st_w(Q4* W, size_t n, size_t k, const Q4& q) {
    double2* p = reinterpret_cast<double2*>(W);
    p[k] = make_double2(q.a, q.b);
    p[n + k] = make_double2(q.c, q.d);
}

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

// compute_dt's per-cell work (solver2d.hpp:74-78) on W = to_primitive(U): non-physical cells are
// recorded, not maxed.
__device__ __forceinline__ void wave_speed_cell(const Q4& W, int lin, double& sx, double& sy, int& bad) {
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
template <int NT>
__device__ __forceinline__ void reduce_wave_speeds(double sx, double sy, int bad, FvCtrl* c, int par) {
    constexpr int NW = NT / 32;
    __shared__ double rsx[NW], rsy[NW];
    __shared__ int rbad[NW];
    sx = warp_max(sx);
    sy = warp_max(sy);
    bad = warp_min_int(bad);
    const int w = threadIdx.x >> 5, l = threadIdx.x & 31;
    if (l == 0) { rsx[w] = sx; rsy[w] = sy; rbad[w] = bad; }
    __syncthreads();
    if (w == 0) {
        sx = l < NW ? rsx[l] : 0.0;
        sy = l < NW ? rsy[l] : 0.0;
        bad = l < NW ? rbad[l] : INT_MAX;
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

// Step control of stage 1, run by one thread per CTA: dt = min(compute_dt(U), t_next - t)
// (main2d.cpp:238, solver2d.hpp:82), or the fixed dt of fv_step.  The leader (one CTA per grid)
// records it for stage 2 and prepares the next reduction slot.  Returns whether the grid steps.
__device__ __forceinline__ bool stage1_control(FvCtrl* c, const GridDesc& g, bool leader, double& dt) {
    const long long step = c->step;
    const int par = int(step & 1);
    const double t = c->t[par];
    bool active = true;
    dt = 0.0;
    if (c->mode == MODE_FIXED) {
        dt = c->dt_fixed;
    } else {
        active = (c->status == 0) && (t < c->t_next);
        if (active && c->bad[par] != INT_MAX) {
            active = false;
            if (leader) {
                c->status = 3;  // FV_ERR_NONPHYSICAL
                c->bad_index = c->bad[par];
            }
        }
        if (active) {
            const double sx = __longlong_as_double((long long)c->sxy[par][0]);
            const double sy = __longlong_as_double((long long)c->sxy[par][1]);
            dt = smin(g.cfl / (sx / g.dx + sy / g.dy), c->t_next - t);
        }
    }
    if (leader) {
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
    return active;
}

// The stage computation of one tile.  STAGE 1: U1 = U + dt L(U).  STAGE 2: U = 0.5 ((U + U1) +
// dt L(U1)), plus the wave speeds of the new U into (sx, sy, bad).
// Step control overlaps the halo load: every thread calls ctl() after issuing its P1 loads (one
// thread does the work and fills the shared `go` and `dt`), and the P1 barrier publishes them.  dt is
// read only in P4.  Returns false (for the whole CTA) when the grid does not step.
// tm: the grid's TMA descriptors for this tile shape, or nullptr; s.bar must have been initialised
// (count 1) by the caller, and `phase` is the barrier's next phase parity (flipped after every TMA
// tile; CTA-uniform).
// Two hooks serve the persistent stepper (fv_stepper.cuh); the per-stage kernels use their defaults:
//  pre4()   -- called by every thread between P3 and P4 (dt is first read in P4); returning false
//              leaves the tile without writing anything (the stepper waits there for the step's dt).
//  COHERENT -- global loads of the stage inputs through L2 (ld.global.cg) instead of the
//              non-coherent / L1 paths, for inputs written earlier in the same launch.
struct NoPre4 {
    __device__ __forceinline__ bool operator()() const { return true; }
};

template <int FLUX, int LIM, int STAGE, int TX, int TY, int NT, class Ctl, class Pre4 = NoPre4, bool COHERENT = false>
__device__ __forceinline__ bool tile_body(const GridDesc& g, const TileMaps* tm, uint32_t& phase, int i0, int j0,
                                          const double& dt, const int& go, Ctl ctl, TileSmem<TX, TY>& s, double& sx,
                                          double& sy, int& bad, Pre4 pre4 = Pre4()) {
    using S = TileSmem<TX, TY>;
    constexpr int HX = S::HX, HY = S::HY;
    constexpr int NSX = TY * (TX + 2), NSY = (TY + 2) * TX;
    constexpr int NFX = TY * (TX + 1), NFY = (TY + 1) * TX;
    const int nx = g.nx, ny = g.ny;
    const size_t ncell = (size_t)nx * ny;
    const Q4* __restrict__ Win = (STAGE == 1) ? g.W : g.W1;

    FV_PHASE_MARK(0);
    // P1: primitives of the halo tile (solver2d.hpp:133-134 on the ghost-filled array).  A tile whose
    // halo lies inside the grid is one TMA box, issued by one thread; a tile at the grid's edge maps
    // every halo cell through the BC.
    const bool tma = tm != nullptr && tm->use && i0 >= 2 && j0 >= 2 && i0 + TX + 2 <= nx && j0 + TY + 2 <= ny &&
                     (tc::smem_addr(&s.W[0][0][0]) & 127u) == 0;  // the copy's destination alignment
    if (tma) {
        if (threadIdx.x == 0) {
            // the CTA's generic accesses to s.W before this point (a previous tile of a persistent
            // CTA, past a CTA barrier) are ordered before the asynchronous proxy's writes
            tc::fence_proxy_async_smem();
            tc::mbar_arrive_expect_tx(&s.bar, (uint32_t)sizeof(s.W));
            tc::tma_load_4d(&s.W[0][0][0], (STAGE == 1) ? (const void*)&tm->w : (const void*)&tm->w1, 0, i0 - 2,
                            j0 - 2, 0, &s.bar);
        }
    } else {
        for (int e = threadIdx.x; e < HX * HY; e += NT) {
            const int r = e / HX, col = e - r * HX;
            const int gi = bc_index(i0 - 2 + col, nx, g.bc_x);
            const int gj = bc_index(j0 - 2 + r, ny, g.bc_y);
            const size_t k = (size_t)gj * nx + gi;
            sts(s.W, r, col, COHERENT ? ldcg_w(Win, ncell, k) : ldg_w(Win, ncell, k));
        }
    }
    ctl();
    __syncthreads();
    if (tma) {  // every thread waits (bounded); the CTA leaves as a whole if any wait ran out
        const int lost = tc::mbar_wait_bounded(&s.bar, phase, nullptr) ? 0 : 1;
        phase ^= 1u;
        if (__syncthreads_or(lost)) {
            if (threadIdx.x == 0) atomicExch(&g.ctrl->status, 4);  // FV_ERR_TIMEOUT: the grid stops
            return false;
        }
    }
    if (!go) return false;
    FV_PHASE_MARK(1);

    // P2: limited slopes.  x-slopes of cells -1..TX per row, y-slopes of rows -1..TY per column.
    auto slope_x = [&](int e) {
        const int r = e / (TX + 2), k = e - r * (TX + 2);  // cell (k-1, r) = W[r+2][k+1]
        sts(s.dX, r, k, limited_slope<LIM>(lds(s.W, r + 2, k), lds(s.W, r + 2, k + 1), lds(s.W, r + 2, k + 2)));
    };
    auto slope_y = [&](int e) {
        const int r = e / TX, k = e - r * TX;  // cell (k, r-1) = W[r+1][k+2]
        sts(s.dY, r, k, limited_slope<LIM>(lds(s.W, r, k + 2), lds(s.W, r + 1, k + 2), lds(s.W, r + 2, k + 2)));
    };
    // Where each direction fits in as many rounds of the CTA's threads as both together, the two
    // directions run as separate loops (uniform code per loop); otherwise as one loop over both.
    if constexpr ((NSX + NT - 1) / NT + (NSY + NT - 1) / NT == (NSX + NSY + NT - 1) / NT) {
        for (int e = threadIdx.x; e < NSX; e += NT) slope_x(e);
        for (int e = threadIdx.x; e < NSY; e += NT) slope_y(e);
    } else {
        for (int e = threadIdx.x; e < NSX + NSY; e += NT) {
            if (e < NSX) slope_x(e);
            else slope_y(e - NSX);
        }
    }
    __syncthreads();
    FV_PHASE_MARK(2);

    // P3: face fluxes, flux(to_conserved(edge(W_L, dW_L, +1)), to_conserved(edge(W_R, dW_R, -1))),
    // with each side's to_primitive by face_side; the y-faces through the momentum swap
    auto face_x = [&](int e) {  // x-face k of row r, between cells k-1 and k (solver2d.hpp:145-148)
        const int r = e / (TX + 1), k = e - r * (TX + 1);
        const FaceSide L = face_side(edge(lds(s.W, r + 2, k + 1), lds(s.dX, r, k), +1.0));
        const FaceSide R = face_side(edge(lds(s.W, r + 2, k + 2), lds(s.dX, r, k + 1), -1.0));
        sts(s.F, r, k, face_flux<FLUX>(L, R));
    };
    auto face_y = [&](int e) {  // y-face r of column k, between rows r-1 and r (solver2d.hpp:165-169)
        const int r = e / TX, k = e - r * TX;
        const FaceSide L = face_side(edge(lds(s.W, r + 1, k + 2), lds(s.dY, r, k), +1.0));
        const FaceSide R = face_side(edge(lds(s.W, r + 2, k + 2), lds(s.dY, r + 1, k), -1.0));
        sts(s.G, r, k, swap_xy(face_flux<FLUX>(swapped(L), swapped(R))));
    };
    if constexpr ((NFX + NT - 1) / NT + (NFY + NT - 1) / NT == (NFX + NFY + NT - 1) / NT) {
        for (int e = threadIdx.x; e < NFX; e += NT) face_x(e);
        for (int e = threadIdx.x; e < NFY; e += NT) face_y(e);
    } else {
        for (int e = threadIdx.x; e < NFX + NFY; e += NT) {
            if (e < NFX) face_x(e);
            else face_y(e - NFX);
        }
    }
    __syncthreads();
    FV_PHASE_MARK(3);
    if (!pre4()) return false;

    // P4: divergence + stage update
    const double cx = g.cx, cy = g.cy;
    for (int e = threadIdx.x; e < TX * TY; e += NT) {
        const int r = e / TX, k = e - r * TX;
        const int i = i0 + k, j = j0 + r;
        if (i >= nx || j >= ny) continue;
        const Q4 Fl = lds(s.F, r, k), Fr = lds(s.F, r, k + 1);
        const Q4 Gb = lds(s.G, r, k), Gt = lds(s.G, r + 1, k);
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
            const Q4 u = COHERENT ? ldcg_q4(g.U + idx) : ldg_q4(g.U + idx);
            const Q4 u1{u.a + dt * L.a, u.b + dt * L.b, u.c + dt * L.c, u.d + dt * L.d};
            st_q4(g.U1 + idx, u1);
            st_w(g.W1, ncell, idx, to_primitive(u1));
        } else {
            const Q4 u = COHERENT ? ldcg_q4(g.U + idx) : ld_q4(g.U + idx);
            const Q4 u1 = COHERENT ? ldcg_q4(g.U1 + idx) : ldg_q4(g.U1 + idx);
            const Q4 un{0.5 * (u.a + u1.a + dt * L.a), 0.5 * (u.b + u1.b + dt * L.b),
                        0.5 * (u.c + u1.c + dt * L.c), 0.5 * (u.d + u1.d + dt * L.d)};
            const Q4 wn = to_primitive(un);
            st_q4(g.U + idx, un);
            st_w(g.W, ncell, idx, wn);
            wave_speed_cell(wn, (int)idx, sx, sy, bad);
        }
    }
    return true;
}

// Single-grid stage kernel: grid (ceil(nx/TX), ceil(ny/TY)), one tile per CTA.
template <int FLUX, int LIM, int STAGE, int TX, int TY, int NT, int MINB>
__global__ void __launch_bounds__(NT, MINB) stage_kernel(const GridDesc g, const __grid_constant__ TileMaps tm) {
    extern __shared__ __align__(128) unsigned char smem_raw[];  // TMA destination: 128-byte aligned
    auto& s = *reinterpret_cast<TileSmem<TX, TY>*>(smem_raw);
    __shared__ double s_dt;
    __shared__ int s_go, s_par2;
    // Programmatic dependent launch: this grid may have been launched while the previous stage still
    // runs; nothing below may touch its outputs before the wait (a no-op for a plain launch).  The
    // next stage may launch once every CTA of this grid has started.
    asm volatile("griddepcontrol.wait;" ::: "memory");
    asm volatile("griddepcontrol.launch_dependents;" :::);
    FvCtrl* c = g.ctrl;
    const bool leader = (blockIdx.x == 0 && blockIdx.y == 0);
    // the last thread has the fewest halo loads: it runs the step control while the others load
    auto ctl = [&]() {
        if (threadIdx.x != NT - 1) return;
        double dt;
        int go, par2 = 0;
        if constexpr (STAGE == 1) {
            go = stage1_control(c, g, leader, dt);
        } else {
            go = c->run2;
            dt = c->dt;
            par2 = c->par2;
        }
        s_go = go; s_dt = dt; s_par2 = par2;
    };
    double sx = 0.0, sy = 0.0;
    int bad = INT_MAX;
    if (tm.use && threadIdx.x == 0) {  // other threads touch the barrier only after the P1 barrier
        tc::mbar_init(&s.bar, 1);
        tc::fence_mbar_init();
    }
    uint32_t phase = 0;
    if (!tile_body<FLUX, LIM, STAGE, TX, TY, NT>(g, &tm, phase, blockIdx.x * TX, blockIdx.y * TY, s_dt, s_go, ctl, s,
                                                 sx, sy, bad))
        return;
    if constexpr (STAGE == 2) {
        reduce_wave_speeds<NT>(sx, sy, bad, c, s_par2);
        if (leader && threadIdx.x == 0) c->step = c->step + 1;
    }
}

// After the state changed from outside the stage kernels: W = to_primitive(U), and the wave speeds /
// positivity of U into slot step&1.
constexpr int RED_NT = 256;
static __global__ void __launch_bounds__(RED_NT) wave_speed_kernel(const Q4* __restrict__ U, Q4* __restrict__ W, int n,
                                                            FvCtrl* c) {
    const int par = int(c->step & 1);
    double sx = 0.0, sy = 0.0;
    int bad = INT_MAX;
    for (int k = blockIdx.x * RED_NT + threadIdx.x; k < n; k += gridDim.x * RED_NT) {
        const Q4 w = to_primitive(ldg_q4(U + k));
        st_w(W, (size_t)n, k, w);
        wave_speed_cell(w, k, sx, sy, bad);
    }
    reduce_wave_speeds<RED_NT>(sx, sy, bad, c, par);
}

static __global__ void ctrl_reset_kernel(FvCtrl* c, double t, int reset_step) {
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

static __global__ void ctrl_set_kernel(FvCtrl* c, int mode, double t_next, double dt_fixed) {
    c->mode = mode;
    c->t_next = t_next;
    c->dt_fixed = dt_fixed;
    if (mode == MODE_LOOP) c->status = 0;
}

static __global__ void ctrl_set_time_kernel(FvCtrl* c, double t) { c->t[int(c->step & 1)] = t; }

// to_conserved of primitive fields (io_hdf5.hpp:197-204); counts cells with !(rho>0)||!(p>0).
static __global__ void primitive_to_state_kernel(const double* __restrict__ rho, const double* __restrict__ u,
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
static __global__ void block_average_kernel(const Q4* __restrict__ U, int nx, int ny, int f, double inv,
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
static __global__ void fill_ghosts_kernel(int nx, int ny, int bc_x, int bc_y, const Q4* __restrict__ U, Q4* __restrict__ Ug) {
    const int W = nx + 4, n = W * (ny + 4);
    for (int k = blockIdx.x * blockDim.x + threadIdx.x; k < n; k += gridDim.x * blockDim.x) {
        const int j = k / W - 2, i = k % W - 2;
        st_q4(Ug + k, ldg_q4(U + (size_t)bc_index(j, ny, bc_y) * nx + bc_index(i, nx, bc_x)));
    }
}

}  // namespace fv
