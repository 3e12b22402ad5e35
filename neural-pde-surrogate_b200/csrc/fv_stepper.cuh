// Persistent dataflow stepper: one cooperative launch advances one grid by many SSP-RK2 steps.
//
// The per-stage kernels (fv_kernels.cuh) launch twice per step, and every launch drains: the last
// tiles of a stage finish at different times while the SMs that finished first sit idle, and the
// next stage starts only when the whole grid is done.  Here a grid of G = (SMs x resident CTAs) CTAs
// stays resident and runs work items in a fixed order:
//     item k  ->  step s = s0 + k / (2T), stage 1 if k mod 2T < T else stage 2, a tile
// (T tiles, visited in row-major order rotated by one tile row per stage).  CTA b runs items
// b, b + G, b + 2G, ... in that order (an ensemble's members share one queue each instead, whose
// items the CTAs claim with an atomic counter).  An item waits only for what it reads or
// overwrites, never for the whole grid:
//   * stage 1 of (s, t) reads U^s, W^s of t and its halo and overwrites U1, W1 of t, which stage 2
//     of step s-1 read: it waits until stage 2 of step s-1 has finished on t's neighbours
//     (flag2[n] >= s for every n in the tile's dependency list: the tiles its halo box maps to,
//     through the boundary conditions, and the tiles whose halo box maps to it);
//   * stage 2 of (s, t) likewise waits for stage 1 of step s on the neighbours (flag1[n] >= s + 1);
//   * the time step is global: dt_s = min(cfl / (sx/dx + sy/dy), t_next - t_s) needs the wave speeds
//     of all of U^s (solver2d.hpp:67-83, main2d.cpp:238).  Stage 1 therefore computes its slopes and
//     face fluxes (phases P1-P3, the bulk of the work) first and waits for the step to be published
//     only before its update (P4); stage 2 waits before it starts.  The last stage-2 item of step s
//     publishes step s + 1 (publish_step), so the next step's first tiles overlap the current step's
//     last ones instead of waiting for a drained grid.
// Every wait ends: an item waits only on items earlier in the order, every CTA runs its items in
// increasing order and all CTAs are co-resident (cooperative launch), so the earliest unfinished
// item is always the one its CTA is running, with every input finished.  Each wait is bounded in
// time all the same (FV_ERR_TIMEOUT, no hang).  An item's completion (flag release, publication)
// runs in one thread while the CTA's next item waits for its inputs and never waits itself.  The arithmetic
// is tile_body's, so results are bit-identical to the per-stage kernels and to the reference.
//
// Memory ordering: a finished item's stores are published by one release store of its flag after
// a CTA barrier (cumulative at GPU scope); a waiting item acquires the flags, then its CTA barrier
// orders every thread's loads after them.  Fields written in the same launch are read through L2
// (tile_body's COHERENT loads) or by TMA, after a proxy fence.
#pragma once
#include "fv_kernels.cuh"

namespace fv {

__device__ __forceinline__ long long ld_acquire(const long long* p) {
    long long v;
    asm volatile("ld.acquire.gpu.global.s64 %0, [%1];" : "=l"(v) : "l"(p) : "memory");
    return v;
}
__device__ __forceinline__ unsigned ld_acquire(const unsigned* p) {
    unsigned v;
    asm volatile("ld.acquire.gpu.global.u32 %0, [%1];" : "=r"(v) : "l"(p) : "memory");
    return v;
}
__device__ __forceinline__ void st_release(long long* p, long long v) {
    asm volatile("st.release.gpu.global.s64 [%0], %1;" ::"l"(p), "l"(v) : "memory");
}
__device__ __forceinline__ void st_release(unsigned* p, unsigned v) {
    asm volatile("st.release.gpu.global.u32 [%0], %1;" ::"l"(p), "r"(v) : "memory");
}
// atomicAdd with release semantics at GPU scope; returns the old value.
__device__ __forceinline__ unsigned long long atom_add_release(unsigned long long* p, unsigned long long v) {
    unsigned long long old;
    asm volatile("atom.release.gpu.global.add.u64 %0, [%1], %2;" : "=l"(old) : "l"(p), "l"(v) : "memory");
    return old;
}
// Orders this thread's generic-proxy view of global memory with its asynchronous-proxy (TMA)
// accesses: W and W1 are written by ordinary stores and read by TMA in the same launch.
__device__ __forceinline__ void fence_proxy_async_global() { asm volatile("fence.proxy.async.global;" ::: "memory"); }

// Tiles of one grid and their dependency lists.  The arrays may hold the tiles of several grids (an
// ensemble): a grid's tile t is entry base + t of the flags and of the compressed rows, whose entries
// dep_idx[dep_off[base + t] .. dep_off[base + t + 1]) are such global tile indices too (built on the
// host by build_stepper_deps).
struct StepperTiles {
    unsigned* flag1;       // per tile: number of steps whose stage 1 has finished on it
    unsigned* flag2;       // per tile: number of steps whose stage 2 has finished on it
    const int* dep_off;
    const int* dep_idx;
    int ntx, nty;          // the grid's tiles
    int base;              // the grid's first tile in the arrays
};

constexpr unsigned long long kStepperWaitNs = 1000000000ull;  // 1 s: far above any legitimate wait

__device__ __forceinline__ int status_now(const FvCtrl* c) { return __ldcg(&c->status); }

// Lane 0 waits until step `target` has been published (c->complete >= target).  Returns false when
// it never will be -- an earlier step does not run (c->stop <= target: t_next reached, a bad cell, or
// the launch's last step) -- on a timeout (recorded as FV_ERR_TIMEOUT), or when another CTA has
// stopped the grid.
__device__ __forceinline__ bool wait_complete(FvCtrl* c, long long target, uint64_t limit_ns = kStepperWaitNs) {
    const uint64_t t0 = tc::globaltimer_ns();
    for (uint32_t it = 0;; ++it) {
        if (ld_acquire(&c->complete) >= target) return true;
        if (__ldcg(&c->stop) <= target) return false;
        if ((it & 15u) == 15u) {
            if (status_now(c) != 0) return false;
            if (tc::globaltimer_ns() - t0 > limit_ns) {
                atomicCAS(&c->status, 0, 4);  // FV_ERR_TIMEOUT
                return false;
            }
            __nanosleep(128);
        }
    }
}

// Warp 0 waits until flag[n] >= target (modulo 2^32) for every dependency n of `tile`.  All 32 lanes
// call it; the result is the same on every lane.
__device__ __forceinline__ bool wait_flags(FvCtrl* c, const unsigned* flag, const StepperTiles& st, int tile,
                                           unsigned target, uint64_t limit_ns = kStepperWaitNs) {
    const int lane = threadIdx.x & 31;
    const int b = st.dep_off[st.base + tile], e = st.dep_off[st.base + tile + 1];
    const uint64_t t0 = tc::globaltimer_ns();
    for (uint32_t it = 0;; ++it) {
        bool mine = true;
        for (int q = b + lane; q < e; q += 32) mine = mine && int(ld_acquire(flag + st.dep_idx[q]) - target) >= 0;
        if (__all_sync(0xffffffffu, mine)) return true;
        if ((it & 15u) == 15u) {
            const bool stop = status_now(c) != 0 || tc::globaltimer_ns() - t0 > limit_ns;
            if (__any_sync(0xffffffffu, stop)) {
                if (lane == 0 && status_now(c) == 0) atomicCAS(&c->status, 0, 4);
                return false;
            }
            __nanosleep(128);
        }
    }
}

// Publication of a completed step j -- every stage-2 item of step j has finished -- or, at the start
// of a launch, of j = s0 - 1 for the state the launch starts from.  From the wave speeds and first bad
// cell of U^{j+1} (reduction slot (j+1) & 1) it decides whether step j+1 runs and with which dt, the
// loop of main2d.cpp:237-242 (dt = min(compute_dt(U), t_next - t)), records t_{j+2}, clears the slot
// that step j+1's stage 2 reduces into, counts the step, and releases c->complete = j.  One thread.
// The decisions are those of stage1_control, so a grid may alternate between the two paths.
__device__ __forceinline__ void publish_step(FvCtrl* c, const GridDesc& g, long long j) {
    const int p1 = int((j + 1) & 1);
    // every input first (independent loads, one round trip), then the decisions
    const double t1 = __ldcg(&c->t[p1]);
    const int status = status_now(c), bad = __ldcg(&c->bad[p1]);
    const double sx = __longlong_as_double((long long)__ldcg(&c->sxy[p1][0]));
    const double sy = __longlong_as_double((long long)__ldcg(&c->sxy[p1][1]));
    const long long s_end = c->s_end;
    const int mode = c->mode;
    const double t_next = c->t_next, dt_fixed = c->dt_fixed;
    bool run = status == 0 && j + 1 < s_end;
    double dt = 0.0;
    if (run) {
        if (mode == MODE_FIXED) {
            dt = dt_fixed;
        } else if (!(t1 < t_next)) {
            run = false;
        } else if (bad != INT_MAX) {
            run = false;
            c->bad_index = bad;
            c->status = 3;  // FV_ERR_NONPHYSICAL
        } else {
            dt = smin(g.cfl / (sx / g.dx + sy / g.dy), t_next - t1);
        }
    }
    c->srun[p1] = run ? 1 : 0;
    c->sdt[p1] = dt;
    if (!run) c->stop = j + 1;  // before the release below: a waiter that sees complete = j sees it
    if (run) {
        c->t[p1 ^ 1] = (mode == MODE_FIXED) ? t1 : t1 + dt;  // fv_step does not advance the time
        c->sxy[p1 ^ 1][0] = 0ull;
        c->sxy[p1 ^ 1][1] = 0ull;
        c->bad[p1 ^ 1] = INT_MAX;
    }
    c->step = j + 1;
    st_release(&c->complete, j);  // release: every write above precedes it
}

// Launch prologue (one small grid before every stepper launch): the queue, the step range, every
// tile's flags set to "all steps before s0 done", and the publication of step s0 - 1.
__device__ __forceinline__ void begin_grid(const GridDesc& g, long long nsteps) {
    FvCtrl* c = g.ctrl;
    const long long s0 = c->step;
    c->queue = 0ull;
    c->done2 = 0ull;
    c->s0 = s0;
    c->s_end = s0 + nsteps;
    c->stop = LLONG_MAX;
    publish_step(c, g, s0 - 1);
}
static __global__ void stepper_begin_kernel(const GridDesc g, StepperTiles st, long long nsteps) {
    const unsigned s0 = unsigned(g.ctrl->step);
    const int T = st.ntx * st.nty;
    for (int t = blockIdx.x * blockDim.x + threadIdx.x; t < T; t += gridDim.x * blockDim.x) {
        st.flag1[st.base + t] = s0;
        st.flag2[st.base + t] = s0;
    }
    if (blockIdx.x == 0 && threadIdx.x == 0) begin_grid(g, nsteps);
}

// Per-CTA state of the item loop, in shared memory.  The current item (step, stage, tile, dt, go) is
// written by lane 0 of warp 0 before the claim barrier.  The previous item's completion runs in two
// threads while warp 0 claims and waits for the next item, so that completion and the next wait
// overlap instead of adding up: thread 32 releases the tile's flag; thread 64, for a stage-2 item,
// adds its block-reduced wave speeds and first bad cell into the next step's slot, counts the item
// and, as the step's last, publishes the step.
struct StepperSlot {
    double dt;
    long long step;
    int go, tile, stage;
    // the grid's launch constants (written by the prologue kernel), read once
    long long s0, s_end;
    double t_next;
    int loop, T;
    // STATIC item sequence: the next item is position r of stage block b (bm = b mod nty); the
    // sequence advances by G = gridDim.x items, i.e. g_blocks blocks and g_rest positions
    long long b;
    int r, bm, g_blocks, g_rest;
    // the last two publications this CTA saw, by the parity of the step j: whether step j + 1 runs,
    // its dt and t_{j+2} (a publication never changes once made)
    long long pub[2];
    int pub_run[2];
    double pub_dt[2], pub_t2[2];
    double red_sx, red_sy;  // the previous stage-2 item's block maxima, its first bad cell
    int red_bad;
    long long prev_step;  // the previous item (prev_stage 0: none)
    int prev_stage, prev_tile;
};
constexpr int kFlagThread = 32, kCountThread = 64;

// Loads grid g's launch constants into the slot and resets its per-grid state; for STATIC items
// also the CTA's first item (blockIdx.x).  One thread, followed by a CTA barrier.
__device__ __forceinline__ void slot_begin(StepperSlot& sl, const GridDesc& g, const StepperTiles& st, bool is_static) {
    const FvCtrl* c = g.ctrl;
    sl.s0 = c->s0;
    sl.s_end = c->s_end;
    sl.t_next = c->t_next;
    sl.loop = c->mode == MODE_LOOP;
    sl.T = st.ntx * st.nty;
    sl.pub[0] = sl.pub[1] = LLONG_MIN;
    sl.prev_stage = 0;
    if (is_static) {
        const unsigned long long T = (unsigned long long)sl.T, G = gridDim.x;
        sl.b = (long long)(blockIdx.x / T);
        sl.r = int(blockIdx.x % T);
        sl.bm = int(sl.b % st.nty);
        sl.g_blocks = int(G / T);
        sl.g_rest = int(G % T);
    }
}

// Lane 0 of warp 0 / thread 0: has step `target` been published (waiting for it, bounded)?  Returns
// the slot entry q (target's parity) whose pub_run[q] / pub_dt[q] / pub_t2[q] hold whether step
// target + 1 runs, its dt and t_{target+2}, or -1 when it never will be (wait_complete).  A CTA asks
// for the same publications for several items, so they are read from L2 once.  The global fields read
// are the ones publish_step(target) wrote: the next write of their parity is publish_step(target + 2),
// which needs the asking item to have finished.
__device__ __forceinline__ int published(FvCtrl* c, StepperSlot& sl, long long target) {
    const int q = int(target & 1);
    if (sl.pub[q] == target) return q;
    if (!wait_complete(c, target)) return -1;
    const int p = int((target + 1) & 1);
    sl.pub_run[q] = __ldcg(&c->srun[p]);
    sl.pub_dt[q] = __ldcg(&c->sdt[p]);
    sl.pub_t2[q] = __ldcg(&c->t[p ^ 1]);
    sl.pub[q] = target;
    return q;
}

// The previous item's completion, after the CTA barrier that follows its stores.  Thread 32: the
// release of the tile's flag (cumulative over the CTA's stores through the barrier).  Thread 64, for
// stage 2: the reduction into slot (step + 1) & 1, then the count (a release: the reduction precedes
// it), and by the step's last item the publication (after an acquire fence: every other item's
// reduction precedes its count, which precedes this one).
__device__ __forceinline__ void release_flag(const StepperTiles& st, const StepperSlot& sl) {
    fence_proxy_async_global();
    unsigned* flag = (sl.prev_stage == 1) ? st.flag1 : st.flag2;
    st_release(flag + st.base + sl.prev_tile, unsigned(sl.prev_step + 1));
}
__device__ __forceinline__ void count_stage2(const GridDesc& g, const StepperSlot& sl) {
    FvCtrl* c = g.ctrl;
    const long long step = sl.prev_step;
    const int par = int((step + 1) & 1);
    if (sl.red_sx > 0.0) atomicMax(&c->sxy[par][0], (unsigned long long)__double_as_longlong(sl.red_sx));
    if (sl.red_sy > 0.0) atomicMax(&c->sxy[par][1], (unsigned long long)__double_as_longlong(sl.red_sy));
    if (sl.red_bad != INT_MAX) atomicMin(&c->bad[par], sl.red_bad);
    const unsigned long long n = atom_add_release(&c->done2, 1ull) + 1ull;
    if (n == (unsigned long long)(step - sl.s0 + 1) * (unsigned long long)sl.T) {
        __threadfence();
        publish_step(c, g, step);
    }
}

// Block maxima of the wave speeds and minimum bad index into sl.red_* (thread 0 writes them); the
// per-stage kernels' reduce_wave_speeds without its global atomics, which count_stage2 issues.
template <int NT>
__device__ __forceinline__ void block_wave_speeds(double sx, double sy, int bad, StepperSlot& sl) {
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
        if (l == 0) { sl.red_sx = sx; sl.red_sy = sy; sl.red_bad = bad; }
    }
}

// Runs grid g's next item: warp 0 takes it (STATIC: the CTA's own sequence blockIdx.x + i gridDim.x;
// else the grid's shared queue) and waits for its inputs, while threads 32 and 64 complete the
// previous item; then the CTA runs the tile body.  Returns false when the grid has no more items to
// run in this launch (past its last step, the loop has reached t_next, a bad cell, or a timeout),
// true after running one.  Called by every thread of the CTA after slot_begin; the mbarrier s.bar
// (when tm is used) is initialised and `phase` tracks it.
template <int FLUX, int LIM, int TX, int TY, int NT, bool STATIC>
__device__ __forceinline__ bool stepper_item(const GridDesc& g, const TileMaps* tm, const StepperTiles& st,
                                             TileSmem<TX, TY>& s, uint32_t& phase, StepperSlot& sl) {
    static_assert(NT > kCountThread, "the completion threads must exist");
    FvCtrl* c = g.ctrl;
    // ---- take the next item and wait for its inputs (warp 0); complete the previous one (32, 64) ----
    if (threadIdx.x < 32) {
        const int lane = threadIdx.x & 31;
        // stage block b (step s0 + b/2, stage 1 + b%2), position r; each block visits the tiles in
        // row-major order starting one tile row further than the block before it (tile r + bm*ntx mod
        // T), so that a block's first rows depend only on the first rows of the block before it
        // (never on its last rows through a periodic wrap)
        long long b;
        int r, bm;
        if constexpr (STATIC) {
            b = sl.b;
            r = sl.r;
            bm = sl.bm;
            __syncwarp();
            if (lane == 0) {  // advance the CTA's sequence by G items
                int r2 = r + sl.g_rest, inc = sl.g_blocks;
                if (r2 >= sl.T) { r2 -= sl.T; ++inc; }
                sl.b = b + inc;
                sl.r = r2;
                sl.bm = int((unsigned)(bm + inc) % (unsigned)st.nty);
            }
        } else {
            unsigned long long k = 0;
            if (lane == 0) k = atomicAdd(&c->queue, 1ull);
            k = __shfl_sync(0xffffffffu, k, 0);
            const unsigned long long T = (unsigned long long)sl.T;
            b = (long long)(k / T);
            r = int(k - (unsigned long long)b * T);
            bm = int(b % st.nty);
        }
        const long long step = sl.s0 + b / 2;
        const int stage = int(b & 1) + 1;
        int tile = r + bm * st.ntx;
        if (tile >= sl.T) tile -= sl.T;
        int go = step < sl.s_end;
        double dt = 0.0;
        if (go && stage == 1) {
            if (step > sl.s0) {
                // step - 1 must run (else nothing will publish its flags) and, in the loop, step
                // must not start at or past t_next; both are known once step - 2 is published
                int ok = 1;
                if (lane == 0) {
                    const int q = published(c, sl, step - 2);
                    ok = q >= 0 && sl.pub_run[q] && (!sl.loop || sl.pub_t2[q] < sl.t_next);
                }
                go = __shfl_sync(0xffffffffu, ok, 0);
                if (go) go = wait_flags(c, st.flag2, st, tile, unsigned(step));
            } else {
                go = __ldcg(&c->srun[sl.s0 & 1]);
            }
        } else if (go) {
            int ok = 1;
            if (lane == 0) {
                const int q = published(c, sl, step - 1);
                ok = q >= 0 && sl.pub_run[q];
                dt = q >= 0 ? sl.pub_dt[q] : 0.0;
            }
            go = __shfl_sync(0xffffffffu, ok, 0);
            if (go) go = wait_flags(c, st.flag1, st, tile, unsigned(step + 1));
        }
        if (lane == 0) {
            if (go) fence_proxy_async_global();  // before this thread issues the tile's TMA load
            sl.go = go;
            sl.step = step;
            sl.stage = stage;
            sl.tile = tile;
            sl.dt = dt;
        }
    } else if (threadIdx.x == kFlagThread) {
        if (sl.prev_stage != 0) release_flag(st, sl);
    } else if (threadIdx.x == kCountThread) {
        if (sl.prev_stage == 2) count_stage2(g, sl);
    }
    __syncthreads();
    if (threadIdx.x == kFlagThread) {  // the item to complete next time, if it runs to its end
        sl.prev_step = sl.step;
        sl.prev_stage = sl.go ? sl.stage : 0;
        sl.prev_tile = sl.tile;
    }
    if (!sl.go) return false;
    const int tyi = sl.tile / st.ntx, txi = sl.tile - tyi * st.ntx;
    double sx = 0.0, sy = 0.0;
    int bad = INT_MAX;
    const int one = 1;
    auto ctl = []() {};
    bool done;
    if (sl.stage == 1) {
        // stage 1 waits for its step's publication only before its update
        auto pre4 = [&]() -> bool {
            if (threadIdx.x == 0) {
                const int q = published(c, sl, sl.step - 1);
                sl.go = q >= 0 && sl.pub_run[q];
                sl.dt = q >= 0 ? sl.pub_dt[q] : 0.0;
            }
            __syncthreads();
            return sl.go != 0;
        };
        done = tile_body<FLUX, LIM, 1, TX, TY, NT, decltype(ctl), decltype(pre4), true>(
            g, tm, phase, txi * TX, tyi * TY, sl.dt, one, ctl, s, sx, sy, bad, pre4);
    } else {
        done = tile_body<FLUX, LIM, 2, TX, TY, NT, decltype(ctl), NoPre4, true>(g, tm, phase, txi * TX, tyi * TY, sl.dt,
                                                                                one, ctl, s, sx, sy, bad);
    }
    if (!done) {  // the step does not run (a bad cell or a timeout stopped the grid): nothing to complete
        if (threadIdx.x == kFlagThread) sl.prev_stage = 0;
        return false;
    }
    if (sl.stage == 2) block_wave_speeds<NT>(sx, sy, bad, sl);  // ends with no barrier
    __syncthreads();  // every store of this item precedes its completion (the next call's)
    return true;
}

// One grid: CTA b runs items b, b + G, b + 2G, ... (G CTAs) in order until it has none left.
template <int FLUX, int LIM, int TX, int TY, int NT, int MINB>
__global__ void __launch_bounds__(NT, MINB) stepper_kernel(const GridDesc g, const __grid_constant__ TileMaps tm,
                                                           const StepperTiles st) {
    extern __shared__ __align__(128) unsigned char smem_raw[];  // TMA destination: 128-byte aligned
    auto& s = *reinterpret_cast<TileSmem<TX, TY>*>(smem_raw);
    __shared__ StepperSlot sl;
    if (threadIdx.x == 0) {
        if (tm.use) {
            tc::mbar_init(&s.bar, 1);
            tc::fence_mbar_init();
        }
        slot_begin(sl, g, st, true);
    }
    __syncthreads();
    uint32_t phase = 0;
    while (stepper_item<FLUX, LIM, TX, TY, NT, true>(g, &tm, st, s, phase, sl)) {
    }
}

// Many grids (an ensemble's members), each with its own queue, control block, dt and t_next.  A CTA
// works on one member until that member has no items left in this launch, then moves to another:
// first member in proportion to the members' tile counts (first[] on the host), then round-robin
// from a shared cursor over the members not yet marked done.  An item still waits only on items of
// its own member claimed before it, each claimed by a resident CTA that finishes it before moving
// on, so every wait ends.  members, tiles and maps (may be NULL) are per-member arrays.
template <int FLUX, int LIM, int TX, int TY, int NT, int MINB>
__global__ void __launch_bounds__(NT, MINB) multi_stepper_kernel(const GridDesc* __restrict__ members,
                                                                 const StepperTiles* __restrict__ tiles,
                                                                 const TileMaps* __restrict__ maps, int count,
                                                                 const int* __restrict__ first, unsigned* member_done,
                                                                 unsigned* cursor) {
    extern __shared__ __align__(128) unsigned char smem_raw[];
    auto& s = *reinterpret_cast<TileSmem<TX, TY>*>(smem_raw);
    __shared__ int s_member;
    __shared__ GridDesc s_g;      // the current member's descriptors, read from shared memory as needed
    __shared__ StepperTiles s_st;
    __shared__ StepperSlot sl;
    if (threadIdx.x == 0) {
        if (maps) {
            tc::mbar_init(&s.bar, 1);
            tc::fence_mbar_init();
        }
        s_member = first[blockIdx.x];
        if (s_member >= 0) {
            s_g = members[s_member];
            s_st = tiles[s_member];
            slot_begin(sl, s_g, s_st, false);
        }
    }
    __syncthreads();
    uint32_t phase = 0;
    for (;;) {
        const int m = s_member;
        if (m < 0) return;
        // a false return leaves nothing to complete (sl.prev_stage 0), so the member may change
        if (!stepper_item<FLUX, LIM, TX, TY, NT, false>(s_g, maps ? maps + m : nullptr, s_st, s, phase, sl)) {
            if (threadIdx.x == 0) {
                atomicExch(member_done + m, 1u);
                const unsigned start = atomicAdd(cursor, 1u);
                int next = -1;
                for (int q = 0; q < count && next < 0; ++q) {
                    const int cand = int((start + unsigned(q)) % unsigned(count));
                    if (ld_acquire(member_done + cand) == 0u) next = cand;
                }
                s_member = next;
                if (next >= 0) {
                    s_g = members[next];
                    s_st = tiles[next];
                    slot_begin(sl, members[next], tiles[next], false);
                }
            }
            __syncthreads();
        }
    }
}

// Launch prologue of the many-grid stepper: every member's queue, step range and publication, every
// tile's flags, the members' done marks and the cursor.
static __global__ void multi_stepper_begin_kernel(const GridDesc* __restrict__ members, const StepperTiles* __restrict__ tiles,
                                           int count, int total_tiles, long long nsteps, unsigned* member_done,
                                           unsigned* cursor) {
    const int stride = gridDim.x * blockDim.x, id = blockIdx.x * blockDim.x + threadIdx.x;
    for (int m = id; m < count; m += stride) {
        const StepperTiles& st = tiles[m];
        const unsigned s0 = unsigned(members[m].ctrl->step);
        for (int t = 0; t < st.ntx * st.nty; ++t) {
            st.flag1[st.base + t] = s0;
            st.flag2[st.base + t] = s0;
        }
        member_done[m] = 0u;
        begin_grid(members[m], nsteps);
    }
    if (id == 0) *cursor = 0u;
    (void)total_tiles;
}

}  // namespace fv
