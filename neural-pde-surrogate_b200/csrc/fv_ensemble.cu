// Batched ensemble: many independent grids (members) of uneven sizes, each with its own CFL dt, time
// and step count, advanced together.  The reference runs one process per trajectory (data/generate.py:
// 60-105, experiments/solver_baseline.py:116-117); here one persistent cooperative launch (the
// many-grid stepper of fv_stepper.cuh) advances every member by many steps to its own target time:
// each member has its own work queue, publication of its dt and tile dependencies, and CTAs move
// between members as their work runs out.  The launch (prologue + stepper) is captured once in a CUDA
// graph and replayed per batch.  With FV_STEPPER=0 the members instead advance by one persistent
// launch per RK stage over the tiles of every running member, replayed in graphs of 16 steps.
//
// Each member's arithmetic is the single-grid tile body with that member's own control block, so
// every member is bit-identical to its own fv_advance_to run.
#include <cuda_runtime.h>

#include <algorithm>
#include <climits>
#include <cmath>
#include <cstring>
#include <vector>

#include "../../include/fv.h"
#include "fv_kernels.cuh"
#include "fv_stepper.cuh"

int fv_internal_set_error(int code, const char* msg);
int fv_internal_encode_maps(const fv::GridDesc& g, int tx, int ty, fv::TileMaps* out);
void fv_internal_stepper_deps(int nx, int ny, int bc_x, int bc_y, int tx, int ty, std::vector<int>& off,
                              std::vector<int>& idx);
bool fv_internal_stepper_enabled();

using namespace fv;

namespace {

constexpr int TX = 16, TY = 14, NT = 256, MINB = 4;  // faces and slopes in two rounds of 256 threads
using Smem = TileSmem<TX, TY>;

struct Tile {
    int member, i0, j0, leader;
};

// One RK stage for every tile of every running member.  Persistent: gridDim.x CTAs stride over the
// tile table.
template <int FLUX, int LIM, int STAGE>
__global__ void __launch_bounds__(NT, MINB) ensemble_stage_kernel(const GridDesc* __restrict__ members,
                                                                  const TileMaps* __restrict__ maps,
                                                                  const Tile* __restrict__ tiles, int ntiles) {
    extern __shared__ __align__(128) unsigned char smem_raw[];  // TMA destination: 128-byte aligned
    Smem& s = *reinterpret_cast<Smem*>(smem_raw);
    __shared__ double s_dt;
    __shared__ int s_go, s_par2;
    // one TMA barrier for all of the CTA's tiles, its phase tracked across them
    if (maps != nullptr && threadIdx.x == 0) {
        tc::mbar_init(&s.bar, 1);
        tc::fence_mbar_init();
    }
    uint32_t phase = 0;
    for (int t = blockIdx.x; t < ntiles; t += gridDim.x) {
        const Tile tile = tiles[t];
        const GridDesc g = members[tile.member];
        FvCtrl* c = g.ctrl;
        if (threadIdx.x == 0) {
            double dt;
            int go, par2 = 0;
            if constexpr (STAGE == 1) {
                go = stage1_control(c, g, tile.leader != 0, dt);
            } else {
                go = c->run2;
                dt = c->dt;
                par2 = c->par2;
            }
            s_go = go; s_dt = dt; s_par2 = par2;
        }
        __syncthreads();
        if (s_go) {
            double sx = 0.0, sy = 0.0;
            int bad = INT_MAX;
            // control ran before the load here: tiles of members that reached their target are skipped
            // without loading anything
            tile_body<FLUX, LIM, STAGE, TX, TY, NT>(g, maps ? maps + tile.member : nullptr, phase, tile.i0, tile.j0,
                                                   s_dt, s_go, [] {}, s, sx, sy, bad);
            if constexpr (STAGE == 2) {
                reduce_wave_speeds<NT>(sx, sy, bad, c, s_par2);
                if (tile.leader && threadIdx.x == 0) c->step = c->step + 1;
            }
        }
        __syncthreads();  // shared memory is reused by the next tile
    }
}

__global__ void ensemble_set_kernel(FvCtrl* ctrl, const double* t_next, int count) {
    const int m = blockIdx.x * blockDim.x + threadIdx.x;
    if (m >= count) return;
    ctrl[m].mode = MODE_LOOP;
    ctrl[m].t_next = t_next[m];
    ctrl[m].status = 0;
}

using StageFn = void (*)(const GridDesc*, const TileMaps*, const Tile*, int);
using MultiFn = void (*)(const GridDesc*, const StepperTiles*, const TileMaps*, int, const int*, unsigned*, unsigned*);

template <int F, int L>
MultiFn multi_of() {
    return multi_stepper_kernel<F, L, TX, TY, NT, MINB>;
}

MultiFn multi_kernel(int flux, int lim) {
    static const MultiFn table[2][4] = {
        {multi_of<0, 0>(), multi_of<0, 1>(), multi_of<0, 2>(), multi_of<0, 3>()},
        {multi_of<1, 0>(), multi_of<1, 1>(), multi_of<1, 2>(), multi_of<1, 3>()}};
    return table[flux][lim];
}

template <int F, int L>
void pick(StageFn* s1, StageFn* s2) {
    *s1 = ensemble_stage_kernel<F, L, 1>;
    *s2 = ensemble_stage_kernel<F, L, 2>;
}

void stage_pair(int flux, int lim, StageFn* s1, StageFn* s2) {
    if (flux == FLUX_HLLC) {
        if (lim == LIM_NONE) pick<FLUX_HLLC, LIM_NONE>(s1, s2);
        else if (lim == LIM_UNLIMITED) pick<FLUX_HLLC, LIM_UNLIMITED>(s1, s2);
        else if (lim == LIM_MINMOD) pick<FLUX_HLLC, LIM_MINMOD>(s1, s2);
        else pick<FLUX_HLLC, LIM_VANLEER>(s1, s2);
    } else {
        if (lim == LIM_NONE) pick<FLUX_RUSANOV, LIM_NONE>(s1, s2);
        else if (lim == LIM_UNLIMITED) pick<FLUX_RUSANOV, LIM_UNLIMITED>(s1, s2);
        else if (lim == LIM_MINMOD) pick<FLUX_RUSANOV, LIM_MINMOD>(s1, s2);
        else pick<FLUX_RUSANOV, LIM_VANLEER>(s1, s2);
    }
}

}  // namespace

struct fv_ensemble {
    int count = 0, flux = 0, lim = 0;
    double cfl = 0.5;
    cudaStream_t stream = nullptr;
    bool own_stream = false;
    std::vector<GridDesc> h_members;   // host copy of the member descriptors
    std::vector<size_t> offset;        // first cell of each member in the state pool
    std::vector<int> has_state;
    size_t total_cells = 0;
    Q4* pool = nullptr;                // U | U1 | W | W1, each total_cells
    FvCtrl* ctrl = nullptr;
    FvCtrl* h_ctrl = nullptr;          // pinned mirror
    GridDesc* d_members = nullptr;
    TileMaps* d_maps = nullptr;        // per member TMA descriptors of W, W1 for the ensemble's tile
    Tile* d_tiles = nullptr;
    int ntiles = 0;
    double* d_tnext = nullptr;
    double* h_tnext = nullptr;         // pinned staging
    StageFn s1 = nullptr, s2 = nullptr;
    int grid = 0;
    cudaGraphExec_t graph = nullptr;   // kGraphSteps ensemble steps
    static constexpr int kGraphSteps = 16;
    long long launches = 0;
    // many-grid stepper: per-member tile tables, all tiles' flags and dependency lists, the first
    // member of every CTA, members' done marks and the cursor (one device allocation)
    MultiFn multi = nullptr;
    void* sbuf = nullptr;
    StepperTiles* d_stiles = nullptr;
    int* d_first = nullptr;
    unsigned* d_done = nullptr;
    unsigned* d_cursor = nullptr;
    int sgrid = 0;
    int total_tiles = 0;
    cudaGraphExec_t sgraph = nullptr;  // prologue + stepper launch of kStepperSteps steps per member
    bool stepper_ready = false;
    static constexpr long long kStepperSteps = 8192;
};

namespace {

int err(int code, const char* msg) { return fv_internal_set_error(code, msg); }

#define EN_CUDA(call)                                                                  \
    do {                                                                               \
        cudaError_t e_ = (call);                                                       \
        if (e_ != cudaSuccess) return err(FV_ERR_CUDA, cudaGetErrorString(e_));        \
    } while (0)

int enqueue_steps(fv_ensemble* e, int nsteps) {
    for (int k = 0; k < nsteps; ++k) {
        e->s1<<<e->grid, NT, sizeof(Smem), e->stream>>>(e->d_members, e->d_maps, e->d_tiles, e->ntiles);
        e->s2<<<e->grid, NT, sizeof(Smem), e->stream>>>(e->d_members, e->d_maps, e->d_tiles, e->ntiles);
    }
    EN_CUDA(cudaGetLastError());
    return FV_OK;
}

int build_graph(fv_ensemble* e) {
    cudaGraph_t g = nullptr;
    EN_CUDA(cudaStreamBeginCapture(e->stream, cudaStreamCaptureModeThreadLocal));
    int rc = enqueue_steps(e, fv_ensemble::kGraphSteps);
    cudaError_t ce = cudaStreamEndCapture(e->stream, &g);
    if (rc) return rc;
    if (ce != cudaSuccess) return err(FV_ERR_CUDA, cudaGetErrorString(ce));
    ce = cudaGraphInstantiate(&e->graph, g, 0);
    cudaGraphDestroy(g);
    if (ce != cudaSuccess) return err(FV_ERR_CUDA, cudaGetErrorString(ce));
    return FV_OK;
}

cudaError_t enqueue_batch(fv_ensemble* e);

// The many-grid stepper's tables (first use): member m's tiles are entries base_m.. of the flags and
// dependency lists, and the CTAs start on the members in proportion to their work.
int prepare_stepper(fv_ensemble* e) {
    e->multi = multi_kernel(e->flux, e->lim);
    EN_CUDA(cudaFuncSetAttribute((const void*)e->multi, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)sizeof(Smem)));
    int per_sm = 0, dev = 0, sms = 0;
    EN_CUDA(cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, e->multi, NT, sizeof(Smem)));
    EN_CUDA(cudaGetDevice(&dev));
    EN_CUDA(cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, dev));
    if (per_sm < 1) return err(FV_ERR_CUDA, "ensemble stepper cannot be resident");
    e->sgrid = per_sm * sms;
    std::vector<StepperTiles> st(e->count);
    std::vector<int> off(1, 0), idx, base(e->count);
    for (int m = 0; m < e->count; ++m) {
        const GridDesc& g = e->h_members[m];
        std::vector<int> o, ix;
        fv_internal_stepper_deps(g.nx, g.ny, g.bc_x, g.bc_y, TX, TY, o, ix);
        base[m] = (int)off.size() - 1;
        const int i0 = (int)idx.size();
        for (int v : ix) idx.push_back(v + base[m]);
        for (size_t t = 1; t < o.size(); ++t) off.push_back(i0 + o[t]);
        st[m] = StepperTiles{nullptr, nullptr, nullptr, nullptr, (g.nx + TX - 1) / TX, (g.ny + TY - 1) / TY, base[m]};
    }
    const int T = (int)off.size() - 1;
    e->total_tiles = T;
    // first member of every CTA, in proportion to the members' work: tiles x steps, and a member's
    // steps to a given time grow with its resolution (CFL), so the weight is tiles x nx
    std::vector<double> cum(e->count + 1, 0.0);
    for (int m = 0; m < e->count; ++m)
        cum[m + 1] = cum[m] + double(st[m].ntx) * st[m].nty * double(e->h_members[m].nx);
    std::vector<int> first(e->sgrid);
    for (int b = 0, m = 0; b < e->sgrid; ++b) {
        const double w = (b + 0.5) * cum[e->count] / e->sgrid;
        while (m + 1 < e->count && cum[m + 1] <= w) ++m;
        first[b] = m;
    }
    const size_t bytes = 2 * size_t(T) * sizeof(unsigned) + (off.size() + idx.size() + first.size()) * sizeof(int) +
                         e->count * (sizeof(StepperTiles) + sizeof(unsigned)) + 2 * sizeof(unsigned) + 64;
    EN_CUDA(cudaMalloc(&e->sbuf, bytes));
    char* p = static_cast<char*>(e->sbuf);
    e->d_stiles = reinterpret_cast<StepperTiles*>(p);  // first: StepperTiles holds pointers (8-byte alignment)
    p += e->count * sizeof(StepperTiles);
    unsigned* flags = reinterpret_cast<unsigned*>(p);
    p += 2 * size_t(T) * sizeof(unsigned);
    int* doff = reinterpret_cast<int*>(p);
    p += off.size() * sizeof(int);
    int* didx = reinterpret_cast<int*>(p);
    p += idx.size() * sizeof(int);
    e->d_first = reinterpret_cast<int*>(p);
    p += first.size() * sizeof(int);
    e->d_done = reinterpret_cast<unsigned*>(p);
    p += e->count * sizeof(unsigned);
    e->d_cursor = reinterpret_cast<unsigned*>(p);
    for (auto& x : st) {
        x.flag1 = flags;
        x.flag2 = flags + T;
        x.dep_off = doff;
        x.dep_idx = didx;
    }
    EN_CUDA(cudaMemcpy(e->d_stiles, st.data(), st.size() * sizeof(StepperTiles), cudaMemcpyHostToDevice));
    EN_CUDA(cudaMemcpy(doff, off.data(), off.size() * sizeof(int), cudaMemcpyHostToDevice));
    EN_CUDA(cudaMemcpy(didx, idx.data(), idx.size() * sizeof(int), cudaMemcpyHostToDevice));
    EN_CUDA(cudaMemcpy(e->d_first, first.data(), first.size() * sizeof(int), cudaMemcpyHostToDevice));
    // the batch launch, captured once: prologue (per-member queues and publications) + stepper; where
    // the runtime cannot capture a cooperative launch, batches are launched directly
    cudaGraph_t gr = nullptr;
    EN_CUDA(cudaStreamBeginCapture(e->stream, cudaStreamCaptureModeThreadLocal));
    cudaError_t ce = enqueue_batch(e);
    cudaError_t ce2 = cudaStreamEndCapture(e->stream, &gr);
    if (ce == cudaSuccess && ce2 == cudaSuccess) ce = cudaGraphInstantiate(&e->sgraph, gr, 0);
    if (gr) cudaGraphDestroy(gr);
    if (ce != cudaSuccess || ce2 != cudaSuccess) {
        e->sgraph = nullptr;
        cudaGetLastError();  // clear the failed capture; the direct launch reports its own errors
    }
    e->stepper_ready = true;
    return FV_OK;
}

// One batch on the stream: prologue + cooperative many-grid stepper.
cudaError_t enqueue_batch(fv_ensemble* e) {
    multi_stepper_begin_kernel<<<std::max(1, std::min((e->count + 127) / 128, 148)), 128, 0, e->stream>>>(
        e->d_members, e->d_stiles, e->count, e->total_tiles, fv_ensemble::kStepperSteps, e->d_done, e->d_cursor);
    cudaError_t ce = cudaGetLastError();
    if (ce != cudaSuccess) return ce;
    cudaLaunchAttribute attr[1];
    attr[0].id = cudaLaunchAttributeCooperative;  // every CTA resident: an item's waits always end
    attr[0].val.cooperative = 1;
    cudaLaunchConfig_t cfg{};
    cfg.gridDim = dim3(e->sgrid);
    cfg.blockDim = dim3(NT);
    cfg.dynamicSmemBytes = sizeof(Smem);
    cfg.stream = e->stream;
    cfg.attrs = attr;
    cfg.numAttrs = 1;
    return cudaLaunchKernelEx(&cfg, e->multi, (const GridDesc*)e->d_members, (const StepperTiles*)e->d_stiles,
                              (const TileMaps*)e->d_maps, e->count, (const int*)e->d_first, e->d_done, e->d_cursor);
}

int read_ctrl(fv_ensemble* e) {
    EN_CUDA(cudaMemcpyAsync(e->h_ctrl, e->ctrl, sizeof(FvCtrl) * e->count, cudaMemcpyDeviceToHost, e->stream));
    EN_CUDA(cudaStreamSynchronize(e->stream));
    return FV_OK;
}

// Every member at once (fv_ensemble_set_all_device): the control blocks reset in one launch, then
// W = to_primitive(U) and the wave speeds / positivity of every member in one launch whose blockIdx.y
// is the member -- instead of two launches per member.  Per member the work and the reduction are
// those of ctrl_reset_kernel + wave_speed_kernel.
__global__ void ensemble_reset_kernel(FvCtrl* ctrl, int count) {
    const int m = blockIdx.x * blockDim.x + threadIdx.x;
    if (m >= count) return;
    FvCtrl* c = ctrl + m;
    c->step = 0;
    c->sxy[0][0] = 0ull;
    c->sxy[0][1] = 0ull;
    c->bad[0] = INT_MAX;
    c->t[0] = 0.0;
    c->status = 0;
    c->bad_index = -1;
    c->run2 = 0;
}
__global__ void __launch_bounds__(RED_NT) ensemble_prime_kernel(const GridDesc* __restrict__ members) {
    const GridDesc g = members[blockIdx.y];
    const int n = g.nx * g.ny;
    double sx = 0.0, sy = 0.0;
    int bad = INT_MAX;
    for (int k = blockIdx.x * RED_NT + threadIdx.x; k < n; k += gridDim.x * RED_NT) {
        const Q4 w = to_primitive(ldg_q4(g.U + k));
        st_w(g.W, (size_t)n, k, w);
        wave_speed_cell(w, k, sx, sy, bad);
    }
    reduce_wave_speeds<RED_NT>(sx, sy, bad, g.ctrl, 0);
}

int prime_member(fv_ensemble* e, int m);

int prime_all(fv_ensemble* e) {
    if (e->count > 65535) {  // beyond gridDim.y: member by member
        for (int m = 0; m < e->count; ++m) {
            int rc = prime_member(e, m);
            if (rc) return rc;
        }
        return FV_OK;
    }
    int maxn = 1;
    for (const GridDesc& g : e->h_members) maxn = std::max(maxn, g.nx * g.ny);
    ensemble_reset_kernel<<<(e->count + 127) / 128, 128, 0, e->stream>>>(e->ctrl, e->count);
    const dim3 grid(std::max(1, std::min((maxn + RED_NT - 1) / RED_NT, 64)), e->count);
    ensemble_prime_kernel<<<grid, RED_NT, 0, e->stream>>>(e->d_members);
    e->launches += 2;
    EN_CUDA(cudaGetLastError());
    for (int m = 0; m < e->count; ++m) e->has_state[m] = 1;
    return FV_OK;
}

int prime_member(fv_ensemble* e, int m) {
    const GridDesc& g = e->h_members[m];
    ctrl_reset_kernel<<<1, 1, 0, e->stream>>>(g.ctrl, 0.0, 1);
    const int n = g.nx * g.ny;
    wave_speed_kernel<<<std::max(1, std::min((n + RED_NT - 1) / RED_NT, 148 * 8)), RED_NT, 0, e->stream>>>(
        g.U, g.W, n, g.ctrl);
    e->launches += 2;
    EN_CUDA(cudaGetLastError());
    e->has_state[m] = 1;
    return FV_OK;
}

}  // namespace

extern "C" {

int fv_ensemble_create(int count, const int* nx, const int* ny, const double* bounds, const int* bc_x,
                       const int* bc_y, int flux, int limiter, double cfl, void* stream, fv_ensemble** out) {
    if (!out || count <= 0 || !nx || !ny || !bc_x || !bc_y) return err(FV_ERR_ARG, "fv_ensemble_create: bad arguments");
    *out = nullptr;
    if ((flux != FLUX_HLLC && flux != FLUX_RUSANOV) || limiter < LIM_NONE || limiter > LIM_VANLEER || !(cfl > 0.0))
        return err(FV_ERR_ARG, "fv_ensemble_create: unknown flux/limiter or bad cfl");
    size_t total = 0;
    for (int m = 0; m < count; ++m) {
        if (nx[m] <= 0 || ny[m] <= 0 || (long long)nx[m] * ny[m] > INT_MAX / 2)
            return err(FV_ERR_ARG, "fv_ensemble_create: member grid sizes must be positive");
        if ((bc_x[m] != BC_PERIODIC && bc_x[m] != BC_TRANSMISSIVE) || (bc_y[m] != BC_PERIODIC && bc_y[m] != BC_TRANSMISSIVE))
            return err(FV_ERR_ARG, "fv_ensemble_create: unknown bc id");
        if (bounds && (!(bounds[4 * m + 1] > bounds[4 * m]) || !(bounds[4 * m + 3] > bounds[4 * m + 2])))
            return err(FV_ERR_ARG, "fv_ensemble_create: empty domain");
        total += size_t(nx[m]) * ny[m];
    }
    int ndev = 0;
    if (cudaGetDeviceCount(&ndev) != cudaSuccess || ndev == 0) return err(FV_ERR_CUDA, "fv_ensemble_create: no CUDA device available");

    fv_ensemble* e = new fv_ensemble;
    e->count = count; e->flux = flux; e->lim = limiter; e->cfl = cfl;
    e->total_cells = total;
    stage_pair(flux, limiter, &e->s1, &e->s2);
    int dev = 0, sms = 148;
    cudaGetDevice(&dev);
    cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, dev);
    e->grid = sms * MINB;
    int rc = FV_OK;
    auto fail = [&](cudaError_t ce) { if (rc == FV_OK) rc = err(FV_ERR_CUDA, cudaGetErrorString(ce)); };
    cudaError_t ce;
    if (stream) e->stream = (cudaStream_t)stream;
    else if ((ce = cudaStreamCreateWithFlags(&e->stream, cudaStreamNonBlocking)) != cudaSuccess) fail(ce);
    else e->own_stream = true;
    if (rc == FV_OK && (ce = cudaMalloc(&e->pool, 4 * total * sizeof(Q4))) != cudaSuccess) fail(ce);
    if (rc == FV_OK && (ce = cudaMalloc(&e->ctrl, count * sizeof(FvCtrl))) != cudaSuccess) fail(ce);
    if (rc == FV_OK && (ce = cudaMallocHost(&e->h_ctrl, count * sizeof(FvCtrl))) != cudaSuccess) fail(ce);
    if (rc == FV_OK && (ce = cudaMalloc(&e->d_members, count * sizeof(GridDesc))) != cudaSuccess) fail(ce);
    if (rc == FV_OK && (ce = cudaMalloc(&e->d_tnext, count * sizeof(double))) != cudaSuccess) fail(ce);
    if (rc == FV_OK && (ce = cudaMallocHost(&e->h_tnext, count * sizeof(double))) != cudaSuccess) fail(ce);
    if (rc == FV_OK && (ce = cudaMemsetAsync(e->ctrl, 0, count * sizeof(FvCtrl), e->stream)) != cudaSuccess) fail(ce);
    std::vector<Tile> tiles;
    if (rc == FV_OK) {
        e->h_members.resize(count);
        e->offset.resize(count);
        e->has_state.assign(count, 0);
        size_t off = 0;
        for (int m = 0; m < count; ++m) {
            GridDesc& g = e->h_members[m];
            const double x0 = bounds ? bounds[4 * m] : 0.0, x1 = bounds ? bounds[4 * m + 1] : 1.0;
            const double y0 = bounds ? bounds[4 * m + 2] : 0.0, y1 = bounds ? bounds[4 * m + 3] : 1.0;
            g.nx = nx[m]; g.ny = ny[m]; g.bc_x = bc_x[m]; g.bc_y = bc_y[m];
            g.dx = (x1 - x0) / nx[m];  // make_grid, grid2d.hpp:34-35
            g.dy = (y1 - y0) / ny[m];
            g.cfl = cfl;
            g.cx = 1.0 / g.dx;
            g.cy = 1.0 / g.dy;
            e->offset[m] = off;
            g.U = e->pool + off;
            g.U1 = e->pool + total + off;
            g.W = e->pool + 2 * total + off;
            g.W1 = e->pool + 3 * total + off;
            g.ctrl = e->ctrl + m;
            off += size_t(nx[m]) * ny[m];
        }
        // tile table, largest members first (they run longest); a member's first tile leads it
        std::vector<int> order(count);
        for (int m = 0; m < count; ++m) order[m] = m;
        std::stable_sort(order.begin(), order.end(), [&](int a, int b) {
            return (long long)nx[a] * ny[a] > (long long)nx[b] * ny[b];
        });
        for (int m : order) {
            bool first = true;
            for (int j0 = 0; j0 < ny[m]; j0 += TY)
                for (int i0 = 0; i0 < nx[m]; i0 += TX) {
                    tiles.push_back(Tile{m, i0, j0, first ? 1 : 0});
                    first = false;
                }
        }
        e->ntiles = (int)tiles.size();
        if ((ce = cudaMalloc(&e->d_tiles, tiles.size() * sizeof(Tile))) != cudaSuccess) fail(ce);
    }
    if (rc == FV_OK && (ce = cudaMemcpy(e->d_tiles, tiles.data(), tiles.size() * sizeof(Tile), cudaMemcpyHostToDevice)) != cudaSuccess) fail(ce);
    if (rc == FV_OK && (ce = cudaMemcpy(e->d_members, e->h_members.data(), count * sizeof(GridDesc), cudaMemcpyHostToDevice)) != cudaSuccess) fail(ce);
    if (rc == FV_OK) {  // TMA descriptors (left out when the driver offers no encoder)
        std::vector<TileMaps> maps(count);
        bool any = false;
        for (int m = 0; m < count && rc == FV_OK; ++m) {
            rc = fv_internal_encode_maps(e->h_members[m], TX, TY, &maps[m]);
            any = any || maps[m].use;
        }
        if (rc == FV_OK && any) {
            if ((ce = cudaMalloc(&e->d_maps, count * sizeof(TileMaps))) != cudaSuccess) fail(ce);
            else if ((ce = cudaMemcpy(e->d_maps, maps.data(), count * sizeof(TileMaps), cudaMemcpyHostToDevice)) != cudaSuccess) fail(ce);
        }
    }
    for (StageFn f : {e->s1, e->s2})
        if (rc == FV_OK && (ce = cudaFuncSetAttribute((const void*)f, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)sizeof(Smem))) != cudaSuccess) fail(ce);
    if (rc != FV_OK) {
        fv_ensemble_destroy(e);
        return rc;
    }
    *out = e;
    return FV_OK;
}

int fv_ensemble_destroy(fv_ensemble* e) {
    if (!e) return FV_OK;
    if (e->stream) cudaStreamSynchronize(e->stream);
    if (e->graph) cudaGraphExecDestroy(e->graph);
    if (e->sgraph) cudaGraphExecDestroy(e->sgraph);
    cudaFree(e->sbuf);
    cudaFree(e->pool);
    cudaFree(e->ctrl);
    cudaFree(e->d_members);
    cudaFree(e->d_maps);
    cudaFree(e->d_tiles);
    cudaFree(e->d_tnext);
    cudaFreeHost(e->h_ctrl);
    cudaFreeHost(e->h_tnext);
    if (e->own_stream && e->stream) cudaStreamDestroy(e->stream);
    delete e;
    return FV_OK;
}

int fv_ensemble_set_state(fv_ensemble* e, int m, const double* U) {
    if (!e || !U || m < 0 || m >= e->count) return err(FV_ERR_ARG, "fv_ensemble_set_state: bad arguments");
    const GridDesc& g = e->h_members[m];
    EN_CUDA(cudaMemcpyAsync(g.U, U, size_t(g.nx) * g.ny * sizeof(Q4), cudaMemcpyHostToDevice, e->stream));
    return prime_member(e, m);
}

int fv_ensemble_set_state_device(fv_ensemble* e, int m, const double* dU) {
    if (!e || !dU || m < 0 || m >= e->count) return err(FV_ERR_ARG, "fv_ensemble_set_state_device: bad arguments");
    const GridDesc& g = e->h_members[m];
    EN_CUDA(cudaMemcpyAsync(g.U, dU, size_t(g.nx) * g.ny * sizeof(Q4), cudaMemcpyDeviceToDevice, e->stream));
    return prime_member(e, m);
}

int fv_ensemble_get_state(fv_ensemble* e, int m, double* U) {
    if (!e || !U || m < 0 || m >= e->count) return err(FV_ERR_ARG, "fv_ensemble_get_state: bad arguments");
    const GridDesc& g = e->h_members[m];
    EN_CUDA(cudaMemcpyAsync(U, g.U, size_t(g.nx) * g.ny * sizeof(Q4), cudaMemcpyDeviceToHost, e->stream));
    EN_CUDA(cudaStreamSynchronize(e->stream));
    return FV_OK;
}

// All members at once from/to one device buffer holding the members' states back to back in member
// order (the ensemble's own pool has exactly that layout).
int fv_ensemble_set_all_device(fv_ensemble* e, const double* dU) {
    if (!e || !dU) return err(FV_ERR_ARG, "fv_ensemble_set_all_device: bad arguments");
    EN_CUDA(cudaMemcpyAsync(e->pool, dU, e->total_cells * sizeof(Q4), cudaMemcpyDeviceToDevice, e->stream));
    return prime_all(e);
}

int fv_ensemble_get_all_device(fv_ensemble* e, double* dU) {
    if (!e || !dU) return err(FV_ERR_ARG, "fv_ensemble_get_all_device: bad arguments");
    EN_CUDA(cudaMemcpyAsync(dU, e->pool, e->total_cells * sizeof(Q4), cudaMemcpyDeviceToDevice, e->stream));
    return FV_OK;
}

int fv_ensemble_state_device(fv_ensemble* e, int m, double** dU) {
    if (!e || !dU || m < 0 || m >= e->count) return err(FV_ERR_ARG, "fv_ensemble_state_device: bad arguments");
    *dU = reinterpret_cast<double*>(e->h_members[m].U);
    return FV_OK;
}

}  // extern "C"

namespace {
// The members' times, step counts and statuses from the control blocks read last.
int finish_advance(fv_ensemble* e, double* t_out, long long* steps_out, int* status_out) {
    int worst = FV_OK;
    for (int m = 0; m < e->count; ++m) {
        const FvCtrl& c = e->h_ctrl[m];
        if (t_out) t_out[m] = c.t[c.step & 1];
        if (steps_out) steps_out[m] = c.step;
        if (status_out) status_out[m] = c.status;
        if (c.status) worst = c.status;
    }
    if (worst == FV_ERR_TIMEOUT) return err(worst, "fv_ensemble_advance_to: a bounded device wait ran out");
    if (worst) return err(worst, "fv_ensemble_advance_to: a member reached a non-physical state (see status)");
    return FV_OK;
}
}  // namespace

extern "C" {

int fv_ensemble_advance_to(fv_ensemble* e, const double* t_next, double* t_out, long long* steps_out, int* status_out) {
    if (!e || !t_next) return err(FV_ERR_ARG, "fv_ensemble_advance_to: bad arguments");
    for (int m = 0; m < e->count; ++m)
        if (!e->has_state[m]) return err(FV_ERR_STATE, "fv_ensemble_advance_to: a member has no state");
    std::memcpy(e->h_tnext, t_next, e->count * sizeof(double));
    EN_CUDA(cudaMemcpyAsync(e->d_tnext, e->h_tnext, e->count * sizeof(double), cudaMemcpyHostToDevice, e->stream));
    ensemble_set_kernel<<<(e->count + 127) / 128, 128, 0, e->stream>>>(e->ctrl, e->d_tnext, e->count);
    e->launches++;
    EN_CUDA(cudaGetLastError());
    int rc = FV_OK;
    if (fv_internal_stepper_enabled()) {
        // one batch (prologue + persistent stepper, a graph replay) advances every member up to
        // kStepperSteps steps towards its target; a member stops by itself at its t_next or a bad cell
        if (!e->stepper_ready && (rc = prepare_stepper(e))) return rc;
        if ((rc = read_ctrl(e))) return rc;
        for (;;) {
            bool more = false;
            for (int m = 0; m < e->count && !more; ++m) {
                const FvCtrl& c = e->h_ctrl[m];
                more = !c.status && c.t[c.step & 1] < t_next[m];
            }
            if (!more) break;
            long long before = 0;
            for (int m = 0; m < e->count; ++m) before += e->h_ctrl[m].step;
            if (e->sgraph) EN_CUDA(cudaGraphLaunch(e->sgraph, e->stream));
            else EN_CUDA(enqueue_batch(e));
            e->launches += 2;
            if ((rc = read_ctrl(e))) return rc;
            long long after = 0;
            for (int m = 0; m < e->count; ++m) after += e->h_ctrl[m].step;
            if (after == before) break;  // nothing could run (the control blocks stopped every member)
        }
        return finish_advance(e, t_out, steps_out, status_out);
    }
    if (!e->graph && (rc = build_graph(e))) return rc;
    if ((rc = read_ctrl(e))) return rc;
    for (;;) {
        // steps still needed by the slowest member, from each member's current CFL dt
        double need = 0.0;
        for (int m = 0; m < e->count; ++m) {
            const FvCtrl& c = e->h_ctrl[m];
            const double t = c.t[c.step & 1];
            if (c.status || !(t < t_next[m])) continue;
            double sx, sy;
            std::memcpy(&sx, &c.sxy[c.step & 1][0], 8);
            std::memcpy(&sy, &c.sxy[c.step & 1][1], 8);
            const GridDesc& g = e->h_members[m];
            const double dt = e->cfl / (sx / g.dx + sy / g.dy);
            need = std::max(need, dt > 0.0 ? std::ceil((t_next[m] - t) / dt) : 1.0);
        }
        if (need <= 0.0) break;
        // whole graph replays (kGraphSteps steps each) while far from the end, single steps near it
        int graphs = (int)std::min(need / fv_ensemble::kGraphSteps, 64.0);
        for (int k = 0; k < graphs; ++k) EN_CUDA(cudaGraphLaunch(e->graph, e->stream));
        e->launches += 2LL * fv_ensemble::kGraphSteps * graphs;
        if (graphs == 0) {
            const int few = (int)std::min(need, (double)fv_ensemble::kGraphSteps);
            if ((rc = enqueue_steps(e, few))) return rc;
            e->launches += 2LL * few;
        }
        if ((rc = read_ctrl(e))) return rc;
    }
    return finish_advance(e, t_out, steps_out, status_out);
}

int fv_ensemble_launch_count(fv_ensemble* e, long long* n) {
    if (!e || !n) return err(FV_ERR_ARG, "fv_ensemble_launch_count: bad arguments");
    *n = e->launches;
    return FV_OK;
}

int fv_ensemble_get_stream(fv_ensemble* e, void** stream) {
    if (!e || !stream) return err(FV_ERR_ARG, "fv_ensemble_get_stream: bad arguments");
    *stream = static_cast<void*>(e->stream);
    return FV_OK;
}

}  // extern "C"
