// C-ABI of the finite-volume solver (include/fv.h): handle management, host<->device copies, the
// device-resident time loop, trajectory output.  No torch types, no exits, no CPU fallback: every
// compute call launches the sm_100a kernels of fv_kernels.cuh.
#include <cuda_runtime.h>

#include <algorithm>
#include <cmath>
#include <cstdarg>
#include <cstdio>
#include <cstdlib>
#include <cstring>
#include <map>
#include <mutex>
#include <set>
#include <string>
#include <tuple>
#include <vector>

#include "../../include/fv.h"
#include "fv_kernels.cuh"
#include "fv_stepper.cuh"

using namespace fv;

namespace {

thread_local std::string g_last_error;

int set_error(int code, const char* fmt, ...) {
    char buf[512];
    va_list ap;
    va_start(ap, fmt);
    vsnprintf(buf, sizeof buf, fmt, ap);
    va_end(ap);
    g_last_error = buf;
    return code;
}

#define FV_CUDA(call)                                                                                  \
    do {                                                                                               \
        cudaError_t e_ = (call);                                                                       \
        if (e_ != cudaSuccess)                                                                         \
            return set_error(FV_ERR_CUDA, "%s failed: %s (%s:%d)", #call, cudaGetErrorString(e_), __FILE__, \
                             __LINE__);                                                                \
    } while (0)

using StageFn = void (*)(GridDesc, TileMaps);

// Tile shapes the stage kernels are instantiated for.  All give bit-identical results; the
// autotuner (fv_autotune) picks the fastest for a grid.  MINB = CTAs per SM the launch bounds ask
// for: NT * MINB = 1024 threads (32 warps) per SM, which caps registers at 64 per thread.
struct TileVariant {
    int tx, ty, nt;
    size_t smem;
    StageFn s1[2][4], s2[2][4];  // [flux][limiter]
};

template <int TX, int TY, int NT, int MINB>
struct VariantMaker {
    template <int F, int L>
    static void one(TileVariant& v) {
        v.s1[F][L] = stage_kernel<F, L, 1, TX, TY, NT, MINB>;
        v.s2[F][L] = stage_kernel<F, L, 2, TX, TY, NT, MINB>;
    }
    static TileVariant make() {
        TileVariant v{TX, TY, NT, sizeof(TileSmem<TX, TY>), {}, {}};
        one<0, 0>(v); one<0, 1>(v); one<0, 2>(v); one<0, 3>(v);
        one<1, 0>(v); one<1, 1>(v); one<1, 2>(v); one<1, 3>(v);
        return v;
    }
};

const std::vector<TileVariant>& variants() {
    static const std::vector<TileVariant> v = {
        VariantMaker<32, 8, 256, 4>::make(),   // 0: default
        VariantMaker<32, 16, 512, 2>::make(),  // 1
        VariantMaker<16, 16, 256, 4>::make(),  // 2
        VariantMaker<64, 8, 512, 2>::make(),   // 3
        VariantMaker<32, 4, 128, 7>::make(),   // 4
        VariantMaker<16, 16, 288, 3>::make(),  // 5: 544 faces over 288 threads -> < 2 rounds
        // shapes whose tile counts fill whole waves (4 x 148 or 2 x 148 resident CTAs) at 512^2 and
        // 256^2, with faces and slopes in two rounds of the CTA's threads
        VariantMaker<16, 14, 256, 4>::make(),  // 6: 512^2 -> 32 x 37 = 1184 tiles = 2 waves of 592
        VariantMaker<32, 14, 512, 2>::make(),  // 7: 512^2 -> 16 x 37 = 592 tiles = 2 waves of 296
        VariantMaker<16, 7, 128, 8>::make(),   // 8: 256^2 -> 16 x 37 = 592 tiles, 8 CTAs per SM
        VariantMaker<16, 14, 256, 5>::make(),  // 9: 40 warps per SM at <= 51 registers
        VariantMaker<16, 7, 128, 9>::make(),   // 10: 36 warps per SM at <= 56 registers
    };
    return v;
}

// Tile shapes the persistent stepper (fv_stepper.cuh) is instantiated for; `variant` is the index of
// the same shape in variants() (whose TMA descriptors it shares).  All give bit-identical results.
using StepperFn = void (*)(GridDesc, TileMaps, StepperTiles);
struct StepperVariant {
    int variant;
    int tx, ty, nt;
    size_t smem;
    StepperFn fn[2][4];  // [flux][limiter]
};

template <int TX, int TY, int NT, int MINB>
struct StepperMaker {
    template <int F, int L>
    static void one(StepperVariant& v) { v.fn[F][L] = stepper_kernel<F, L, TX, TY, NT, MINB>; }
    static StepperVariant make(int variant) {
        StepperVariant v{variant, TX, TY, NT, sizeof(TileSmem<TX, TY>), {}};
        one<0, 0>(v); one<0, 1>(v); one<0, 2>(v); one<0, 3>(v);
        one<1, 0>(v); one<1, 1>(v); one<1, 2>(v); one<1, 3>(v);
        return v;
    }
};

const std::vector<StepperVariant>& stepper_variants() {
    static const std::vector<StepperVariant> v = {
        StepperMaker<16, 14, 256, 4>::make(6),  // 0: default
        StepperMaker<16, 16, 256, 4>::make(2),  // 1
        StepperMaker<32, 8, 256, 4>::make(0),   // 2
        StepperMaker<16, 7, 128, 8>::make(8),   // 3
        StepperMaker<32, 16, 512, 2>::make(1),  // 4
        StepperMaker<16, 7, 128, 9>::make(10),  // 5: 36 warps per SM at <= 56 registers
        StepperMaker<32, 14, 512, 2>::make(7),  // 6: 512^2 -> 592 tiles, exactly 2 per CTA and stage
    };
    return v;
}

// Autotuned choice per (device, nx, ny, flux, limiter), shared by all handles of the process.
std::mutex g_tune_mu;
std::map<std::tuple<int, int, int, int, int>, int> g_tuned;
std::map<std::tuple<int, int, int, int, int>, int> g_tuned_stepper;

// Host copy of bc_index (fv_physics.cuh) for the stepper's dependency lists.
int host_bc_index(int g, int n, int bc) {
    if (bc == BC_PERIODIC) {
        const int m = g % n;
        return m < 0 ? m + n : m;
    }
    return g < 0 ? 0 : (g >= n ? n - 1 : g);
}

// The stepper's dependency list of every tile: the tiles that hold a cell of its halo box
// [i0 - 2, i0 + tx + 1] x [j0 - 2, j0 + ty + 1] once mapped through the boundary conditions (whose
// stage outputs it reads), and the tiles whose halo box holds one of its cells (which read what it
// overwrites), itself included.  Compressed rows: off has ntx*nty + 1 entries.
void build_stepper_deps(int nx, int ny, int bc_x, int bc_y, int tx, int ty, std::vector<int>& off,
                        std::vector<int>& idx) {
    const int ntx = (nx + tx - 1) / tx, nty = (ny + ty - 1) / ty, T = ntx * nty;
    auto axis = [](int t, int w, int n, int bc) {
        std::set<int> out;
        for (int c = t * w - 2; c <= t * w + w + 1; ++c) out.insert(host_bc_index(c, n, bc) / w);
        return out;
    };
    std::vector<std::set<int>> deps(T);
    for (int b = 0; b < nty; ++b) {
        const std::set<int> ys = axis(b, ty, ny, bc_y);
        for (int a = 0; a < ntx; ++a) {
            const std::set<int> xs = axis(a, tx, nx, bc_x);
            const int t = b * ntx + a;
            for (int y : ys)
                for (int x : xs) {
                    const int d = y * ntx + x;
                    deps[t].insert(d);  // t reads d
                    deps[d].insert(t);  // d overwrites what t reads
                }
        }
    }
    off.assign(1, 0);
    idx.clear();
    for (int t = 0; t < T; ++t) {
        deps[t].insert(t);
        idx.insert(idx.end(), deps[t].begin(), deps[t].end());
        off.push_back((int)idx.size());
    }
}

}  // namespace

struct fv_solver {
    int nx = 0, ny = 0, bc_x = 0, bc_y = 0, flux = 0, lim = 0;
    double x_min = 0, x_max = 1, y_min = 0, y_max = 1, dx = 0, dy = 0, cfl = 0.5;
    int device = 0;
    cudaStream_t stream = nullptr;
    bool own_stream = false;
    Q4* U = nullptr;
    Q4* U1 = nullptr;
    Q4* W = nullptr;   // to_primitive(U), kept current by every kernel that writes U
    Q4* W1 = nullptr;  // to_primitive(U1)
    FvCtrl* ctrl = nullptr;
    FvCtrl* h_ctrl = nullptr;  // pinned mirror
    int* d_count = nullptr;
    int* h_count = nullptr;
    double* d_prim = nullptr;  // staging for fv_set_primitive (4 * n doubles), allocated on first use
    float* d_avg = nullptr;
    size_t d_avg_cap = 0;
    int variant = 0;          // tile shape (index into variants())
    TileMaps maps{};          // TMA descriptors of W, W1 for the tile shape maps_variant
    int maps_variant = -1;
    bool tuned = false;       // variant chosen by the autotuner or fixed by fv_set_tile
    bool has_state = false;
    long long launches = 0;  // kernels launched by this handle
    // kernel timing (fv_profile): a ring of event triples bracketing stage 1 and stage 2
    static constexpr int kRing = 256;
    bool profiling = false;
    cudaEvent_t ev[kRing][3] = {};
    int ring_head = 0, ring_used = 0;
    double ms1 = 0.0, ms2 = 0.0;
    long long timed = 0;
    // persistent stepper: tile shape (index into stepper_variants(), -1 before the first choice), its
    // TMA descriptors, flags and dependency lists (one device allocation), and its timing
    int svariant = -1;
    bool stuned = false;
    TileMaps smaps{};
    int smaps_variant = -1;
    void* sbuf = nullptr;
    int sbuf_variant = -1;
    StepperTiles st{};
    int sgrid = 0;          // co-resident CTAs of the chosen stepper kernel
    cudaEvent_t sev[2] = {};
    double step_ms = 0.0;   // stepper launches' device time since fv_profile(1) (all kernels of a launch)
    long long step_steps = 0, step_launches = 0;

    size_t ncell() const { return size_t(nx) * ny; }
    GridDesc desc() const {
        GridDesc g{};
        g.U = U; g.U1 = U1; g.W = W; g.W1 = W1;
        g.nx = nx; g.ny = ny; g.bc_x = bc_x; g.bc_y = bc_y;
        g.dx = dx; g.dy = dy; g.cfl = cfl;
        g.cx = 1.0 / dx; g.cy = 1.0 / dy;  // (1.0 / g.dx) of solver2d.hpp:149-150
        g.ctrl = ctrl;
        return g;
    }
};

namespace {

int retire_oldest(fv_solver* s) {
    cudaEvent_t* ev = s->ev[s->ring_head];
    FV_CUDA(cudaEventSynchronize(ev[2]));
    float a = 0.f, b = 0.f;
    FV_CUDA(cudaEventElapsedTime(&a, ev[0], ev[1]));
    FV_CUDA(cudaEventElapsedTime(&b, ev[1], ev[2]));
    s->ms1 += a;
    s->ms2 += b;
    s->timed++;
    s->ring_head = (s->ring_head + 1) % fv_solver::kRing;
    s->ring_used--;
    return FV_OK;
}

// cuTensorMapEncodeTiled from the driver, looked up once through the runtime (no link to libcuda).
using EncodeTiledFn = CUresult (*)(CUtensorMap*, CUtensorMapDataType, cuuint32_t, void*, const cuuint64_t*,
                                   const cuuint64_t*, const cuuint32_t*, const cuuint32_t*, CUtensorMapInterleave,
                                   CUtensorMapSwizzle, CUtensorMapL2promotion, CUtensorMapFloatOOBfill);
EncodeTiledFn encode_tiled() {
    static EncodeTiledFn fn = [] {
        void* p = nullptr;
        cudaDriverEntryPointQueryResult q;
        if (cudaGetDriverEntryPoint("cuTensorMapEncodeTiled", &p, cudaEnableDefault, &q) != cudaSuccess ||
            q != cudaDriverEntryPointSuccess)
            p = nullptr;
        return reinterpret_cast<EncodeTiledFn>(p);
    }();
    return fn;
}

// TMA descriptors of g's primitive arrays (two planes of nx*ny double2 each) for a (tx+4) x (ty+4)
// halo box.  use = 0 when the driver offers no encoder (every tile then takes the BC-mapped load).
int encode_maps(const GridDesc& g, int tx, int ty, TileMaps* out) {
    *out = TileMaps{};
    EncodeTiledFn fn = encode_tiled();
    if (!fn) return FV_OK;
    const cuuint64_t dims[4] = {2, (cuuint64_t)g.nx, (cuuint64_t)g.ny, 2};
    const cuuint64_t strides[3] = {16, 16ull * g.nx, 16ull * g.nx * g.ny};  // bytes, dims 1..3
    const cuuint32_t box[4] = {2, (cuuint32_t)(tx + 4), (cuuint32_t)(ty + 4), 2};
    const cuuint32_t estr[4] = {1, 1, 1, 1};
    for (int k = 0; k < 2; ++k) {
        CUresult r = fn(k == 0 ? &out->w : &out->w1, CU_TENSOR_MAP_DATA_TYPE_FLOAT64, 4, k == 0 ? (void*)g.W : (void*)g.W1,
                        dims, strides, box, estr, CU_TENSOR_MAP_INTERLEAVE_NONE, CU_TENSOR_MAP_SWIZZLE_NONE,
                        CU_TENSOR_MAP_L2_PROMOTION_L2_128B, CU_TENSOR_MAP_FLOAT_OOB_FILL_NONE);
        if (r != CUDA_SUCCESS) return set_error(FV_ERR_CUDA, "cuTensorMapEncodeTiled failed (%d)", (int)r);
    }
    out->use = 1;
    return FV_OK;
}

// Enqueues stage 1 and stage 2 of one step of grid g with tile variant v.
int enqueue_step(const GridDesc& g, const TileMaps& tm, int v, int flux, int lim, cudaStream_t st, cudaEvent_t* ev) {
    const TileVariant& tv = variants()[v];
    const dim3 grid((g.nx + tv.tx - 1) / tv.tx, (g.ny + tv.ty - 1) / tv.ty);
    // both stages as programmatic dependent launches: a stage's CTAs get resident while the previous
    // kernel of the stream drains, and start the moment it completes (griddepcontrol.wait)
    cudaLaunchAttribute attr[1];
    attr[0].id = cudaLaunchAttributeProgrammaticStreamSerialization;
    attr[0].val.programmaticStreamSerializationAllowed = 1;
    cudaLaunchConfig_t cfg{};
    cfg.gridDim = grid;
    cfg.blockDim = dim3(tv.nt);
    cfg.dynamicSmemBytes = tv.smem;
    cfg.stream = st;
    cfg.attrs = attr;
    cfg.numAttrs = 1;  // with events between the stages, each interval is completion to completion
    if (ev) FV_CUDA(cudaEventRecord(ev[0], st));
    FV_CUDA(cudaLaunchKernelEx(&cfg, tv.s1[flux][lim], g, tm));
    if (ev) FV_CUDA(cudaEventRecord(ev[1], st));
    FV_CUDA(cudaLaunchKernelEx(&cfg, tv.s2[flux][lim], g, tm));
    if (ev) FV_CUDA(cudaEventRecord(ev[2], st));
    FV_CUDA(cudaGetLastError());
    return FV_OK;
}

int prepare_variants(int flux, int lim) {
    static std::mutex mu;
    static bool done[2][4] = {};
    std::lock_guard<std::mutex> lock(mu);
    if (done[flux][lim]) return FV_OK;
    for (const TileVariant& v : variants()) {
        for (StageFn f : {v.s1[flux][lim], v.s2[flux][lim]})
            FV_CUDA(cudaFuncSetAttribute((const void*)f, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)v.smem));
    }
    done[flux][lim] = true;
    return FV_OK;
}

int autotune(fv_solver* s, int steps, int* chosen);

int launch_step(fv_solver* s) {
    if (!s->tuned) {
        int rc = autotune(s, 8, nullptr);
        if (rc) return rc;
    }
    cudaEvent_t* ev = nullptr;
    if (s->profiling) {
        if (s->ring_used == fv_solver::kRing) {  // retire the oldest triple before reusing it
            int rc = retire_oldest(s);
            if (rc) return rc;
        }
        ev = s->ev[(s->ring_head + s->ring_used) % fv_solver::kRing];
        s->ring_used++;
    }
    s->launches += 2;
    if (s->maps_variant != s->variant) {
        const TileVariant& tv = variants()[s->variant];
        int rc = encode_maps(s->desc(), tv.tx, tv.ty, &s->maps);
        if (rc) return rc;
        s->maps_variant = s->variant;
    }
    return enqueue_step(s->desc(), s->maps, s->variant, s->flux, s->lim, s->stream, ev);
}

int read_ctrl(fv_solver* s) {
    FV_CUDA(cudaMemcpyAsync(s->h_ctrl, s->ctrl, sizeof(FvCtrl), cudaMemcpyDeviceToHost, s->stream));
    FV_CUDA(cudaStreamSynchronize(s->stream));
    return FV_OK;
}

// Reads the cell of a recorded bad index and fills *bad the way report_bad_cell prints it.
int fill_bad(fv_solver* s, int lin, fv_bad_cell* bad) {
    if (!bad) return FV_OK;
    double q[4];
    FV_CUDA(cudaMemcpyAsync(q, s->U + lin, sizeof q, cudaMemcpyDeviceToHost, s->stream));
    FV_CUDA(cudaStreamSynchronize(s->stream));
    const double u = q[1] / q[0], v = q[2] / q[0];
    bad->i = lin % s->nx;
    bad->j = lin / s->nx;
    bad->rho = q[0];
    bad->p = GM1 * (q[3] - 0.5 * q[0] * (u * u + v * v));
    return FV_OK;
}

// After the state changed from the host: reset the control block and reduce the wave speeds.
int prime_state(fv_solver* s, double t, bool reset_step) {
    ctrl_reset_kernel<<<1, 1, 0, s->stream>>>(s->ctrl, t, reset_step ? 1 : 0);
    const int n = int(s->ncell());
    const int blocks = std::max(1, std::min((n + RED_NT - 1) / RED_NT, 148 * 8));
    wave_speed_kernel<<<blocks, RED_NT, 0, s->stream>>>(s->U, s->W, n, s->ctrl);
    s->launches += 2;
    FV_CUDA(cudaGetLastError());
    s->has_state = true;
    return FV_OK;
}

// Times every tile variant on a copy of the current state (fixed dt from the current CFL dt, so the
// handle's state, time and control block are untouched) and keeps the fastest.
int autotune(fv_solver* s, int steps, int* chosen) {
    s->tuned = true;  // also on failure: never retried inside launch_step
    const auto key = std::make_tuple(s->device, s->nx, s->ny, s->flux, s->lim);
    if (!chosen) {
        std::lock_guard<std::mutex> lock(g_tune_mu);
        auto it = g_tuned.find(key);
        if (it != g_tuned.end()) {
            s->variant = it->second;
            return FV_OK;
        }
    }
    if (!s->has_state) return FV_OK;  // nothing to time on yet: keep the default shape
    double dt = 1e-6;
    {
        int rc = read_ctrl(s);
        if (rc) return rc;
        const FvCtrl& c = *s->h_ctrl;
        double sx, sy;
        std::memcpy(&sx, &c.sxy[c.step & 1][0], 8);
        std::memcpy(&sy, &c.sxy[c.step & 1][1], 8);
        const double d = s->cfl / (sx / s->dx + sy / s->dy);
        if (d > 0.0 && std::isfinite(d)) dt = d;
    }
    const size_t bytes = s->ncell() * sizeof(Q4);
    Q4* tmp = nullptr;  // copies of U, U1, W, W1
    FvCtrl* ct = nullptr;
    cudaEvent_t e0 = nullptr, e1 = nullptr;
    int rc = FV_OK, best = s->variant;
    float best_ms = 1e30f;
    cudaError_t e = cudaMalloc(&tmp, 4 * bytes);
    if (e == cudaSuccess) e = cudaMalloc(&ct, sizeof(FvCtrl));
    if (e == cudaSuccess) e = cudaEventCreate(&e0);
    if (e == cudaSuccess) e = cudaEventCreate(&e1);
    const size_t n = s->ncell();
    for (int v = 0; e == cudaSuccess && v < (int)variants().size(); ++v) {
        GridDesc g = s->desc();
        g.U = tmp; g.U1 = tmp + n; g.W = tmp + 2 * n; g.W1 = tmp + 3 * n; g.ctrl = ct;
        e = cudaMemcpyAsync(g.U, s->U, bytes, cudaMemcpyDeviceToDevice, s->stream);
        if (e == cudaSuccess) e = cudaMemcpyAsync(g.W, s->W, bytes, cudaMemcpyDeviceToDevice, s->stream);
        if (e != cudaSuccess) break;
        ctrl_reset_kernel<<<1, 1, 0, s->stream>>>(ct, 0.0, 1);
        ctrl_set_kernel<<<1, 1, 0, s->stream>>>(ct, MODE_FIXED, 0.0, dt);
        TileMaps tm;
        if ((rc = encode_maps(g, variants()[v].tx, variants()[v].ty, &tm))) break;
        for (int k = 0; k < 2 && rc == FV_OK; ++k) rc = enqueue_step(g, tm, v, s->flux, s->lim, s->stream, nullptr);
        if (rc) break;
        if ((e = cudaEventRecord(e0, s->stream)) != cudaSuccess) break;
        for (int k = 0; k < steps && rc == FV_OK; ++k) rc = enqueue_step(g, tm, v, s->flux, s->lim, s->stream, nullptr);
        if (rc) break;
        if ((e = cudaEventRecord(e1, s->stream)) != cudaSuccess) break;
        if ((e = cudaEventSynchronize(e1)) != cudaSuccess) break;
        float ms = 0.f;
        if ((e = cudaEventElapsedTime(&ms, e0, e1)) != cudaSuccess) break;
        s->launches += 2 * (steps + 2) + 2;
        if (ms < best_ms) { best_ms = ms; best = v; }
    }
    if (e0) cudaEventDestroy(e0);
    if (e1) cudaEventDestroy(e1);
    cudaFree(tmp);
    cudaFree(ct);
    if (rc) return rc;
    if (e != cudaSuccess) return set_error(FV_ERR_CUDA, "fv_autotune: %s", cudaGetErrorString(e));
    s->variant = best;
    if (chosen) *chosen = best;
    std::lock_guard<std::mutex> lock(g_tune_mu);
    g_tuned[key] = best;
    return FV_OK;
}

// ---- persistent stepper (fv_stepper.cuh) --------------------------------------------------------

// FV_STEPPER=0 in the environment keeps fv_advance_to on the per-stage kernels (for comparisons).
bool stepper_enabled() {
    static const bool on = [] {
        const char* e = getenv("FV_STEPPER");
        return !(e && atoi(e) == 0);
    }();
    return on;
}

// Readies stepper shape sv for the handle: kernel attributes and co-residency (cached per kernel),
// the flags and dependency lists of the handle's grid (one device allocation, rebuilt when the shape
// changes) and the TMA descriptors of the shape.
int prepare_stepper(fv_solver* s, int sv) {
    const StepperVariant& v = stepper_variants()[sv];
    StepperFn fn = v.fn[s->flux][s->lim];
    static std::mutex mu;
    static std::map<std::pair<int, StepperFn>, int> resident;
    int per_sm = 0;
    {
        std::lock_guard<std::mutex> lock(mu);
        auto it = resident.find({s->device, fn});
        if (it == resident.end()) {
            FV_CUDA(cudaFuncSetAttribute((const void*)fn, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)v.smem));
            FV_CUDA(cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, fn, v.nt, v.smem));
            resident[{s->device, fn}] = per_sm;
        } else {
            per_sm = it->second;
        }
    }
    int sms = 0;
    FV_CUDA(cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, s->device));
    if (per_sm < 1) return set_error(FV_ERR_CUDA, "stepper tile %dx%d cannot be resident", v.tx, v.ty);
    if (s->sbuf_variant != sv) {
        std::vector<int> off, idx;
        build_stepper_deps(s->nx, s->ny, s->bc_x, s->bc_y, v.tx, v.ty, off, idx);
        const size_t T = off.size() - 1;
        cudaFree(s->sbuf);
        s->sbuf = nullptr;
        s->sbuf_variant = -1;
        FV_CUDA(cudaMalloc(&s->sbuf, 2 * T * sizeof(unsigned) + (off.size() + idx.size()) * sizeof(int)));
        unsigned* flags = static_cast<unsigned*>(s->sbuf);
        int* doff = reinterpret_cast<int*>(flags + 2 * T);
        int* didx = doff + off.size();
        FV_CUDA(cudaMemcpyAsync(doff, off.data(), off.size() * sizeof(int), cudaMemcpyHostToDevice, s->stream));
        FV_CUDA(cudaMemcpyAsync(didx, idx.data(), idx.size() * sizeof(int), cudaMemcpyHostToDevice, s->stream));
        FV_CUDA(cudaStreamSynchronize(s->stream));  // the host vectors go out of scope
        s->st = StepperTiles{flags, flags + T, doff, didx, (s->nx + v.tx - 1) / v.tx, (s->ny + v.ty - 1) / v.ty};
        s->sbuf_variant = sv;
    }
    if (s->smaps_variant != v.variant) {
        int rc = encode_maps(s->desc(), v.tx, v.ty, &s->smaps);
        if (rc) return rc;
        s->smaps_variant = v.variant;
    }
    s->sgrid = per_sm * sms;
    return FV_OK;
}

// One stepper launch on grid g: the prologue kernel (queue, flags, publication of the current step)
// and the cooperative kernel, which runs at most nsteps steps and stops by itself where the loop
// reaches t_next, a bad cell appears, or a bounded wait runs out.
int enqueue_stepper(const GridDesc& g, const TileMaps& tm, const StepperTiles& st, int sv, int flux, int lim,
                    int grid, long long nsteps, cudaStream_t stream) {
    const StepperVariant& v = stepper_variants()[sv];
    const long long T = (long long)st.ntx * st.nty;
    stepper_begin_kernel<<<(unsigned)std::max<long long>(1, std::min<long long>((T + 255) / 256, 148)), 256, 0, stream>>>(
        g, st, nsteps);
    FV_CUDA(cudaGetLastError());
    cudaLaunchAttribute attr[1];
    attr[0].id = cudaLaunchAttributeCooperative;  // every CTA resident: an item's waits always end
    attr[0].val.cooperative = 1;
    cudaLaunchConfig_t cfg{};
    cfg.gridDim = dim3((unsigned)std::min<long long>(grid, 2 * T * nsteps));
    cfg.blockDim = dim3(v.nt);
    cfg.dynamicSmemBytes = v.smem;
    cfg.stream = stream;
    cfg.attrs = attr;
    cfg.numAttrs = 1;
    FV_CUDA(cudaLaunchKernelEx(&cfg, v.fn[flux][lim], g, tm, st));
    return FV_OK;
}

// Times every stepper shape for `steps` fixed-dt steps on copies of the current state (the handle's
// state, time and control block are untouched) and keeps the fastest: the persistent counterpart of
// autotune().  FV_STEPPER_TILE=<index> fixes the shape instead.
int autotune_stepper(fv_solver* s, int steps) {
    s->stuned = true;
    s->svariant = 0;
    const auto key = std::make_tuple(s->device, s->nx, s->ny, s->flux, s->lim);
    const char* env = getenv("FV_STEPPER_TILE");
    if (env && atoi(env) >= 0 && atoi(env) < (int)stepper_variants().size()) {
        s->svariant = atoi(env);
        return FV_OK;
    }
    {
        std::lock_guard<std::mutex> lock(g_tune_mu);
        auto it = g_tuned_stepper.find(key);
        if (it != g_tuned_stepper.end()) {
            s->svariant = it->second;
            return FV_OK;
        }
    }
    if (!s->has_state) return FV_OK;
    double dt = 1e-6;
    int rc = read_ctrl(s);
    if (rc) return rc;
    {
        const FvCtrl& c = *s->h_ctrl;
        double sx, sy;
        std::memcpy(&sx, &c.sxy[c.step & 1][0], 8);
        std::memcpy(&sy, &c.sxy[c.step & 1][1], 8);
        const double d = s->cfl / (sx / s->dx + sy / s->dy);
        if (d > 0.0 && std::isfinite(d)) dt = d;
    }
    const size_t n = s->ncell(), bytes = n * sizeof(Q4);
    Q4* tmp = nullptr;
    FvCtrl* ct = nullptr;
    cudaEvent_t e0 = nullptr, e1 = nullptr;
    int best = 0;
    float best_ms = 1e30f;
    cudaError_t e = cudaMalloc(&tmp, 4 * bytes);
    if (e == cudaSuccess) e = cudaMalloc(&ct, sizeof(FvCtrl));
    if (e == cudaSuccess) e = cudaEventCreate(&e0);
    if (e == cudaSuccess) e = cudaEventCreate(&e1);
    for (int v = 0; e == cudaSuccess && rc == FV_OK && v < (int)stepper_variants().size(); ++v) {
        if ((rc = prepare_stepper(s, v))) break;
        GridDesc g = s->desc();
        g.U = tmp; g.U1 = tmp + n; g.W = tmp + 2 * n; g.W1 = tmp + 3 * n; g.ctrl = ct;
        TileMaps tm;
        if ((rc = encode_maps(g, stepper_variants()[v].tx, stepper_variants()[v].ty, &tm))) break;
        float ms = 0.f;
        for (int pass = 0; pass < 2 && rc == FV_OK && e == cudaSuccess; ++pass) {  // pass 0 warms up
            e = cudaMemcpyAsync(g.U, s->U, bytes, cudaMemcpyDeviceToDevice, s->stream);
            if (e == cudaSuccess) e = cudaMemcpyAsync(g.W, s->W, bytes, cudaMemcpyDeviceToDevice, s->stream);
            if (e == cudaSuccess) e = cudaMemcpyAsync(ct, s->ctrl, sizeof(FvCtrl), cudaMemcpyDeviceToDevice, s->stream);
            if (e != cudaSuccess) break;
            ctrl_set_kernel<<<1, 1, 0, s->stream>>>(ct, MODE_FIXED, 0.0, dt);
            ctrl_reset_kernel<<<1, 1, 0, s->stream>>>(ct, 0.0, 1);  // clears any status of the copy
            if ((e = cudaEventRecord(e0, s->stream)) != cudaSuccess) break;
            rc = enqueue_stepper(g, tm, s->st, v, s->flux, s->lim, s->sgrid, pass ? steps : 2, s->stream);
            if (rc) break;
            if ((e = cudaEventRecord(e1, s->stream)) != cudaSuccess) break;
            if ((e = cudaEventSynchronize(e1)) != cudaSuccess) break;
            if ((e = cudaEventElapsedTime(&ms, e0, e1)) != cudaSuccess) break;
            s->launches += 4;
        }
        if (rc == FV_OK && e == cudaSuccess && ms < best_ms) {
            best_ms = ms;
            best = v;
        }
    }
    if (e0) cudaEventDestroy(e0);
    if (e1) cudaEventDestroy(e1);
    cudaFree(tmp);
    cudaFree(ct);
    if (rc) return rc;
    if (e != cudaSuccess) return set_error(FV_ERR_CUDA, "stepper autotune: %s", cudaGetErrorString(e));
    s->svariant = best;
    std::lock_guard<std::mutex> lock(g_tune_mu);
    g_tuned_stepper[key] = best;
    return FV_OK;
}

// fv_advance_to on the persistent stepper: one launch per batch of up to 4096 steps (the kernel
// stops by itself at t_next), the control block read once per launch.  The control block has been
// set to loop mode and read into h_ctrl by the caller.
int advance_stepper(fv_solver* s, double t_next) {
    if (!s->stuned) {
        int rc = autotune_stepper(s, 8);
        if (rc) return rc;
    }
    int rc = prepare_stepper(s, s->svariant);
    if (rc) return rc;
    for (;;) {
        const FvCtrl& c = *s->h_ctrl;
        if (c.status) break;
        const double t = c.t[c.step & 1];
        if (!(t < t_next)) break;
        double sx, sy;
        std::memcpy(&sx, &c.sxy[c.step & 1][0], 8);
        std::memcpy(&sy, &c.sxy[c.step & 1][1], 8);
        const double dt_est = s->cfl / (sx / s->dx + sy / s->dy);
        const double est = (dt_est > 0.0) ? std::ceil((t_next - t) / dt_est) : 1.0;
        const long long nsteps = (long long)std::min(4096.0, std::max(1.0, 2.0 * est + 16.0));
        const long long before = c.step;
        if (s->profiling) FV_CUDA(cudaEventRecord(s->sev[0], s->stream));
        if ((rc = enqueue_stepper(s->desc(), s->smaps, s->st, s->svariant, s->flux, s->lim, s->sgrid, nsteps,
                                  s->stream)))
            return rc;
        s->launches += 2;
        if (s->profiling) FV_CUDA(cudaEventRecord(s->sev[1], s->stream));
        if ((rc = read_ctrl(s))) return rc;
        if (s->profiling) {
            float ms = 0.f;
            FV_CUDA(cudaEventElapsedTime(&ms, s->sev[0], s->sev[1]));
            s->step_ms += ms;
            s->step_steps += s->h_ctrl->step - before;
            s->step_launches++;
        }
        if (s->h_ctrl->step == before) break;  // nothing ran (the control block stopped the grid)
    }
    return FV_OK;
}

bool valid_common(int flux, int lim, int bc_x, int bc_y) {
    return (flux == FLUX_HLLC || flux == FLUX_RUSANOV) && lim >= LIM_NONE && lim <= LIM_VANLEER &&
           (bc_x == BC_PERIODIC || bc_x == BC_TRANSMISSIVE) && (bc_y == BC_PERIODIC || bc_y == BC_TRANSMISSIVE);
}

}  // namespace

// Lets the library's other translation units report through fv_last_error().
int fv_internal_set_error(int code, const char* msg) { return set_error(code, "%s", msg ? msg : ""); }
int fv_internal_encode_maps(const GridDesc& g, int tx, int ty, TileMaps* out) { return encode_maps(g, tx, ty, out); }
void fv_internal_stepper_deps(int nx, int ny, int bc_x, int bc_y, int tx, int ty, std::vector<int>& off,
                              std::vector<int>& idx) {
    build_stepper_deps(nx, ny, bc_x, bc_y, tx, ty, off, idx);
}
bool fv_internal_stepper_enabled() { return stepper_enabled(); }

extern "C" {

const char* fv_last_error(void) { return g_last_error.c_str(); }
#ifdef FV_TOLERANCE_BUILD
const char* fv_version(void) { return "fv-b200 1.0 (sm_100a, FP64, tolerance build: FMA contraction)"; }
#else
const char* fv_version(void) { return "fv-b200 1.0 (sm_100a, FP64, bit-exact build)"; }
#endif

int fv_create(int nx, int ny, double x_min, double x_max, double y_min, double y_max, int bc_x, int bc_y,
              int flux, int limiter, double cfl, void* stream, fv_solver** out) {
    if (!out) return set_error(FV_ERR_ARG, "fv_create: out is NULL");
    *out = nullptr;
    if (nx <= 0 || ny <= 0) return set_error(FV_ERR_ARG, "fv_create: nx and ny must be positive");
    if ((long long)nx * ny > (long long)INT_MAX / 2) return set_error(FV_ERR_ARG, "fv_create: grid too large");
    if (!(cfl > 0.0)) return set_error(FV_ERR_ARG, "fv_create: cfl must be positive");
    if (!(x_max > x_min) || !(y_max > y_min)) return set_error(FV_ERR_ARG, "fv_create: empty domain");
    if (!valid_common(flux, limiter, bc_x, bc_y)) return set_error(FV_ERR_ARG, "fv_create: unknown flux/limiter/bc id");
    int ndev = 0;
    if (cudaGetDeviceCount(&ndev) != cudaSuccess || ndev == 0)
        return set_error(FV_ERR_CUDA, "fv_create: no CUDA device available");

    fv_solver* s = new fv_solver;
    s->nx = nx; s->ny = ny; s->bc_x = bc_x; s->bc_y = bc_y; s->flux = flux; s->lim = limiter;
    s->x_min = x_min; s->x_max = x_max; s->y_min = y_min; s->y_max = y_max;
    s->dx = (x_max - x_min) / nx;  // make_grid, grid2d.hpp:34-35
    s->dy = (y_max - y_min) / ny;
    s->cfl = cfl;
    cudaGetDevice(&s->device);
    int rc = FV_OK;
    auto fail = [&](cudaError_t e, const char* what) {
        rc = set_error(FV_ERR_CUDA, "fv_create: %s: %s", what, cudaGetErrorString(e));
    };
    cudaError_t e;
    if (stream) {
        s->stream = (cudaStream_t)stream;
    } else if ((e = cudaStreamCreateWithFlags(&s->stream, cudaStreamNonBlocking)) != cudaSuccess) {
        fail(e, "stream");
    } else {
        s->own_stream = true;
    }
    if (rc == FV_OK && (e = cudaMalloc(&s->U, s->ncell() * sizeof(Q4))) != cudaSuccess) fail(e, "state");
    if (rc == FV_OK && (e = cudaMalloc(&s->U1, s->ncell() * sizeof(Q4))) != cudaSuccess) fail(e, "stage state");
    if (rc == FV_OK && (e = cudaMalloc(&s->W, s->ncell() * sizeof(Q4))) != cudaSuccess) fail(e, "primitives");
    if (rc == FV_OK && (e = cudaMalloc(&s->W1, s->ncell() * sizeof(Q4))) != cudaSuccess) fail(e, "stage primitives");
    if (rc == FV_OK && (e = cudaMalloc(&s->ctrl, sizeof(FvCtrl))) != cudaSuccess) fail(e, "control block");
    if (rc == FV_OK && (e = cudaMalloc(&s->d_count, sizeof(int))) != cudaSuccess) fail(e, "counter");
    if (rc == FV_OK && (e = cudaMallocHost(&s->h_ctrl, sizeof(FvCtrl))) != cudaSuccess) fail(e, "pinned control");
    if (rc == FV_OK && (e = cudaMallocHost(&s->h_count, sizeof(int))) != cudaSuccess) fail(e, "pinned counter");
    if (rc == FV_OK && (e = cudaMemsetAsync(s->ctrl, 0, sizeof(FvCtrl), s->stream)) != cudaSuccess) fail(e, "memset");
    if (rc == FV_OK) rc = prepare_variants(flux, limiter);
    if (rc == FV_OK) {
        std::lock_guard<std::mutex> lock(g_tune_mu);
        auto it = g_tuned.find({s->device, nx, ny, flux, limiter});
        const char* env = getenv("FV_TILE");
        const char* at = getenv("FV_AUTOTUNE");
        if (env && atoi(env) >= 0 && atoi(env) < (int)variants().size()) {  // fixed tile shape
            s->variant = atoi(env);
            s->tuned = true;
        } else if (it != g_tuned.end()) {
            s->variant = it->second;
            s->tuned = true;
        } else if (at && atoi(at) == 0) {
            s->tuned = true;  // keep the default variant
        }
    }
    if (rc != FV_OK) {
        fv_destroy(s);
        return rc;
    }
    *out = s;
    return FV_OK;
}

int fv_destroy(fv_solver* s) {
    if (!s) return FV_OK;
    if (s->stream) cudaStreamSynchronize(s->stream);
    for (auto& tri : s->ev)
        for (cudaEvent_t& e : tri)
            if (e) cudaEventDestroy(e);
    for (cudaEvent_t& e : s->sev)
        if (e) cudaEventDestroy(e);
    cudaFree(s->sbuf);
    cudaFree(s->U);
    cudaFree(s->U1);
    cudaFree(s->W);
    cudaFree(s->W1);
    cudaFree(s->ctrl);
    cudaFree(s->d_count);
    cudaFree(s->d_prim);
    cudaFree(s->d_avg);
    cudaFreeHost(s->h_ctrl);
    cudaFreeHost(s->h_count);
    if (s->own_stream && s->stream) cudaStreamDestroy(s->stream);
    delete s;
    return FV_OK;
}

int fv_set_state(fv_solver* s, const double* U) {
    if (!s || !U) return set_error(FV_ERR_ARG, "fv_set_state: NULL argument");
    FV_CUDA(cudaMemcpyAsync(s->U, U, s->ncell() * sizeof(Q4), cudaMemcpyHostToDevice, s->stream));
    return prime_state(s, 0.0, true);
}

int fv_set_state_device(fv_solver* s, const double* dU) {
    if (!s || !dU) return set_error(FV_ERR_ARG, "fv_set_state_device: NULL argument");
    FV_CUDA(cudaMemcpyAsync(s->U, dU, s->ncell() * sizeof(Q4), cudaMemcpyDeviceToDevice, s->stream));
    return prime_state(s, 0.0, true);
}

int fv_get_state(fv_solver* s, double* U) {
    if (!s || !U) return set_error(FV_ERR_ARG, "fv_get_state: NULL argument");
    FV_CUDA(cudaMemcpyAsync(U, s->U, s->ncell() * sizeof(Q4), cudaMemcpyDeviceToHost, s->stream));
    FV_CUDA(cudaStreamSynchronize(s->stream));
    return FV_OK;
}

int fv_get_state_device(fv_solver* s, double* dU) {
    if (!s || !dU) return set_error(FV_ERR_ARG, "fv_get_state_device: NULL argument");
    FV_CUDA(cudaMemcpyAsync(dU, s->U, s->ncell() * sizeof(Q4), cudaMemcpyDeviceToDevice, s->stream));
    return FV_OK;
}

int fv_set_primitive(fv_solver* s, const double* rho, const double* u, const double* v, const double* p) {
    if (!s || !rho || !u || !v || !p) return set_error(FV_ERR_ARG, "fv_set_primitive: NULL argument");
    const size_t n = s->ncell();
    if (!s->d_prim) FV_CUDA(cudaMalloc(&s->d_prim, 4 * n * sizeof(double)));
    const double* src[4] = {rho, u, v, p};
    for (int q = 0; q < 4; ++q)
        FV_CUDA(cudaMemcpyAsync(s->d_prim + q * n, src[q], n * sizeof(double), cudaMemcpyHostToDevice, s->stream));
    // Convert into U1 first so that a rejected input leaves the state unchanged.
    FV_CUDA(cudaMemsetAsync(s->d_count, 0, sizeof(int), s->stream));
    s->launches++;
    primitive_to_state_kernel<<<std::max(1, std::min(int((n + 255) / 256), 148 * 8)), 256, 0, s->stream>>>(
        s->d_prim, s->d_prim + n, s->d_prim + 2 * n, s->d_prim + 3 * n, int(n), s->U1, s->d_count);
    FV_CUDA(cudaGetLastError());
    FV_CUDA(cudaMemcpyAsync(s->h_count, s->d_count, sizeof(int), cudaMemcpyDeviceToHost, s->stream));
    FV_CUDA(cudaStreamSynchronize(s->stream));
    if (*s->h_count)
        return set_error(FV_ERR_ARG, "initial condition has non-positive density or pressure (%d cells)", *s->h_count);
    FV_CUDA(cudaMemcpyAsync(s->U, s->U1, n * sizeof(Q4), cudaMemcpyDeviceToDevice, s->stream));
    return prime_state(s, 0.0, true);
}

int fv_set_time(fv_solver* s, double t) {
    if (!s) return set_error(FV_ERR_ARG, "fv_set_time: NULL handle");
    ctrl_set_time_kernel<<<1, 1, 0, s->stream>>>(s->ctrl, t);
    s->launches++;
    FV_CUDA(cudaGetLastError());
    return FV_OK;
}

int fv_get_time(fv_solver* s, double* t, long long* steps) {
    if (!s) return set_error(FV_ERR_ARG, "fv_get_time: NULL handle");
    int rc = read_ctrl(s);
    if (rc) return rc;
    if (t) *t = s->h_ctrl->t[s->h_ctrl->step & 1];
    if (steps) *steps = s->h_ctrl->step;
    return FV_OK;
}

int fv_compute_dt(fv_solver* s, double* dt, fv_bad_cell* bad) {
    if (!s || !dt) return set_error(FV_ERR_ARG, "fv_compute_dt: NULL argument");
    if (!s->has_state) return set_error(FV_ERR_STATE, "fv_compute_dt: no state set");
    int rc = read_ctrl(s);
    if (rc) return rc;
    const FvCtrl& c = *s->h_ctrl;
    const int par = int(c.step & 1);
    if (c.bad[par] != INT_MAX) {
        fill_bad(s, c.bad[par], bad);
        return set_error(FV_ERR_NONPHYSICAL, "Non-physical state in cell (%d, %d)", c.bad[par] % s->nx,
                         c.bad[par] / s->nx);
    }
    double sx, sy;
    std::memcpy(&sx, &c.sxy[par][0], 8);
    std::memcpy(&sy, &c.sxy[par][1], 8);
    *dt = s->cfl / (sx / s->dx + sy / s->dy);  // solver2d.hpp:82
    return FV_OK;
}

int fv_step(fv_solver* s, double dt) {
    if (!s) return set_error(FV_ERR_ARG, "fv_step: NULL handle");
    if (!s->has_state) return set_error(FV_ERR_STATE, "fv_step: no state set");
    ctrl_set_kernel<<<1, 1, 0, s->stream>>>(s->ctrl, MODE_FIXED, 0.0, dt);
    s->launches++;
    return launch_step(s);
}

int fv_advance_to(fv_solver* s, double t_next, double* t_out, long long* steps_out, fv_bad_cell* bad) {
    if (!s) return set_error(FV_ERR_ARG, "fv_advance_to: NULL handle");
    if (!s->has_state) return set_error(FV_ERR_STATE, "fv_advance_to: no state set");
    ctrl_set_kernel<<<1, 1, 0, s->stream>>>(s->ctrl, MODE_LOOP, t_next, 0.0);
    s->launches++;
    FV_CUDA(cudaGetLastError());
    int rc = read_ctrl(s);
    if (rc) return rc;
    if (stepper_enabled()) {
        if ((rc = advance_stepper(s, t_next))) return rc;
    }
    // Per-stage kernels: steps are queued in batches sized from the last dt; steps queued after t
    // reaches t_next (or after a non-physical state) exit at their first instruction, so a batch may
    // overshoot freely.
    const int kMaxBatch = 256;
    for (;;) {
        const FvCtrl& c = *s->h_ctrl;
        if (c.status) break;
        const double t = c.t[c.step & 1];
        if (!(t < t_next)) break;
        // CFL dt of the current state (the last dt of a frame is clamped to land on it, so it is
        // useless as an estimate); the remaining steps are estimated from it without overshoot.
        double sx, sy;
        std::memcpy(&sx, &c.sxy[c.step & 1][0], 8);
        std::memcpy(&sy, &c.sxy[c.step & 1][1], 8);
        const double dt_est = s->cfl / (sx / s->dx + sy / s->dy);
        double est = (dt_est > 0.0) ? std::ceil((t_next - t) / dt_est) : 1.0;
        int batch = (int)std::min<double>(std::max(est, 1.0), (double)kMaxBatch);
        for (int k = 0; k < batch; ++k)
            if ((rc = launch_step(s))) return rc;
        if ((rc = read_ctrl(s))) return rc;
    }
    const FvCtrl& c = *s->h_ctrl;
    if (t_out) *t_out = c.t[c.step & 1];
    if (steps_out) *steps_out = c.step;
    if (c.status == FV_ERR_NONPHYSICAL) {
        fill_bad(s, c.bad_index, bad);
        return set_error(FV_ERR_NONPHYSICAL, "Non-physical state in cell (%d, %d)", c.bad_index % s->nx,
                         c.bad_index / s->nx);
    }
    if (c.status == FV_ERR_TIMEOUT)
        return set_error(FV_ERR_TIMEOUT, "fv_advance_to: a bounded device wait ran out (a tile's TMA load or a "
                                         "stepper dependency)");
    return FV_OK;
}

int fv_block_average_device(fv_solver* s, int f, float* d_out) {
    if (!s || !d_out) return set_error(FV_ERR_ARG, "fv_block_average: NULL argument");
    if (f <= 0 || s->nx % f || s->ny % f)
        return set_error(FV_ERR_ARG, "save factor %d does not divide the %d x %d grid", f, s->nx, s->ny);
    const int n = (s->nx / f) * (s->ny / f);
    const double inv = 1.0 / (double(f) * f);  // trajectory.hpp:34
    s->launches++;
    block_average_kernel<<<std::max(1, std::min((n + 255) / 256, 148 * 8)), 256, 0, s->stream>>>(
        s->U, s->nx, s->ny, f, inv, d_out);
    FV_CUDA(cudaGetLastError());
    return FV_OK;
}

int fv_block_average(fv_solver* s, int f, float* out) {
    if (!s || !out) return set_error(FV_ERR_ARG, "fv_block_average: NULL argument");
    if (f <= 0 || s->nx % f || s->ny % f)
        return set_error(FV_ERR_ARG, "save factor %d does not divide the %d x %d grid", f, s->nx, s->ny);
    const size_t n = size_t(4) * (s->nx / f) * (s->ny / f);
    if (s->d_avg_cap < n) {
        cudaFree(s->d_avg);
        s->d_avg = nullptr;
        s->d_avg_cap = 0;
        FV_CUDA(cudaMalloc(&s->d_avg, n * sizeof(float)));
        s->d_avg_cap = n;
    }
    int rc = fv_block_average_device(s, f, s->d_avg);
    if (rc) return rc;
    FV_CUDA(cudaMemcpyAsync(out, s->d_avg, n * sizeof(float), cudaMemcpyDeviceToHost, s->stream));
    FV_CUDA(cudaStreamSynchronize(s->stream));
    return FV_OK;
}

int fv_run_trajectory(fv_solver* s, double t_start, double t_end, int nout, const int* sizes, int nsizes,
                      float** out, double* times, long long* steps, fv_bad_cell* bad) {
    if (!s) return set_error(FV_ERR_ARG, "fv_run_trajectory: NULL handle");
    if (nout <= 0) return set_error(FV_ERR_ARG, "n, nout and cfl must be positive");
    if (!(t_end > 0.0)) return set_error(FV_ERR_ARG, "tend must be positive");
    if (!(t_start >= 0.0 && t_start < t_end)) return set_error(FV_ERR_ARG, "need 0 <= tstart < t_end");
    if (nsizes < 0 || (nsizes > 0 && (!sizes || !out))) return set_error(FV_ERR_ARG, "fv_run_trajectory: bad sizes");
    std::vector<int> factors;
    for (int l = 0; l < nsizes; ++l) {  // TrajectoryWriter ctor checks, trajectory.hpp:19-28
        const int m = sizes[l];
        if (m <= 0 || s->nx % m != 0) return set_error(FV_ERR_ARG, "save size %d does not divide nx = %d", m, s->nx);
        const int f = s->nx / m;
        if (s->ny % f != 0) return set_error(FV_ERR_ARG, "save size %d does not divide ny evenly", m);
        factors.push_back(f);
    }
    double t = 0.0;
    long long nst = 0;
    auto output = [&](int k) -> int {
        if (times) times[k] = t;
        for (int l = 0; l < nsizes; ++l) {
            const int f = factors[l];
            const size_t frame = size_t(4) * (s->nx / f) * (s->ny / f);
            int rc = fv_block_average(s, f, out[l] + size_t(k) * frame);
            if (rc) return rc;
        }
        return FV_OK;
    };
    int rc = fv_get_time(s, &t, &nst);
    if (rc) return rc;
    if (t < t_start && (rc = fv_advance_to(s, t_start, &t, &nst, bad))) return rc;  // main2d.cpp:227-232
    if ((rc = output(0))) return rc;
    for (int k = 1; k <= nout; ++k) {
        const double t_next = t_start + (t_end - t_start) * k / nout;  // main2d.cpp:236
        if ((rc = fv_advance_to(s, t_next, &t, &nst, bad))) return rc;
        if ((rc = output(k))) return rc;
    }
    if (steps) *steps = nst;
    return FV_OK;
}

int fv_riemann_flux(int flux, int y_face, int n, const double* UL, const double* UR, double* F) {
    if (n < 0 || (n > 0 && (!UL || !UR || !F))) return set_error(FV_ERR_ARG, "fv_riemann_flux: bad arguments");
    if (flux != FLUX_HLLC && flux != FLUX_RUSANOV) return set_error(FV_ERR_ARG, "fv_riemann_flux: unknown flux");
    if (n == 0) return FV_OK;
    Q4* d = nullptr;
    const size_t bytes = size_t(n) * sizeof(Q4);
    FV_CUDA(cudaMalloc(&d, 3 * bytes));
    cudaError_t e = cudaMemcpy(d, UL, bytes, cudaMemcpyHostToDevice);
    if (e == cudaSuccess) e = cudaMemcpy(d + n, UR, bytes, cudaMemcpyHostToDevice);
    if (e == cudaSuccess) {
        const int blocks = std::min((n + 127) / 128, 1024);
        if (flux == FLUX_HLLC) riemann_flux_kernel<FLUX_HLLC><<<blocks, 128>>>(n, y_face, d, d + n, d + 2 * n);
        else riemann_flux_kernel<FLUX_RUSANOV><<<blocks, 128>>>(n, y_face, d, d + n, d + 2 * n);
        e = cudaGetLastError();
    }
    if (e == cudaSuccess) e = cudaMemcpy(F, d + 2 * n, bytes, cudaMemcpyDeviceToHost);
    cudaFree(d);
    if (e != cudaSuccess) return set_error(FV_ERR_CUDA, "fv_riemann_flux: %s", cudaGetErrorString(e));
    return FV_OK;
}

}  // extern "C"

// q[k] = a[k] / b[k] by the division every general division site of the stage kernels uses (fdiv).
static __global__ void division_kernel(int n, const double* __restrict__ a, const double* __restrict__ b,
                                       double* __restrict__ q) {
    for (int k = blockIdx.x * blockDim.x + threadIdx.x; k < n; k += gridDim.x * blockDim.x) q[k] = fv::fdiv(a[k], b[k]);
}

extern "C" {

int fv_eval_division(int n, const double* a, const double* b, double* q) {
    if (n < 0 || (n > 0 && (!a || !b || !q))) return set_error(FV_ERR_ARG, "fv_eval_division: bad arguments");
    if (n == 0) return FV_OK;
    double* d = nullptr;
    const size_t bytes = size_t(n) * sizeof(double);
    FV_CUDA(cudaMalloc(&d, 3 * bytes));
    cudaError_t e = cudaMemcpy(d, a, bytes, cudaMemcpyHostToDevice);
    if (e == cudaSuccess) e = cudaMemcpy(d + n, b, bytes, cudaMemcpyHostToDevice);
    if (e == cudaSuccess) {
        division_kernel<<<std::min((n + 255) / 256, 148 * 8), 256>>>(n, d, d + n, d + 2 * n);
        e = cudaGetLastError();
    }
    if (e == cudaSuccess) e = cudaMemcpy(q, d + 2 * n, bytes, cudaMemcpyDeviceToHost);
    cudaFree(d);
    if (e != cudaSuccess) return set_error(FV_ERR_CUDA, "fv_eval_division: %s", cudaGetErrorString(e));
    return FV_OK;
}

int fv_fill_ghosts(int nx, int ny, int bc_x, int bc_y, const double* U, double* Ug) {
    if (nx <= 0 || ny <= 0 || !U || !Ug) return set_error(FV_ERR_ARG, "fv_fill_ghosts: bad arguments");
    if (!valid_common(FLUX_HLLC, LIM_NONE, bc_x, bc_y)) return set_error(FV_ERR_ARG, "fv_fill_ghosts: unknown bc");
    const size_t n_in = size_t(nx) * ny, n_out = size_t(nx + 4) * (ny + 4);
    Q4* d = nullptr;
    FV_CUDA(cudaMalloc(&d, (n_in + n_out) * sizeof(Q4)));
    cudaError_t e = cudaMemcpy(d, U, n_in * sizeof(Q4), cudaMemcpyHostToDevice);
    if (e == cudaSuccess) {
        fill_ghosts_kernel<<<int(std::min<size_t>((n_out + 127) / 128, 1024)), 128>>>(nx, ny, bc_x, bc_y, d, d + n_in);
        e = cudaGetLastError();
    }
    if (e == cudaSuccess) e = cudaMemcpy(Ug, d + n_in, n_out * sizeof(Q4), cudaMemcpyDeviceToHost);
    cudaFree(d);
    if (e != cudaSuccess) return set_error(FV_ERR_CUDA, "fv_fill_ghosts: %s", cudaGetErrorString(e));
    return FV_OK;
}

int fv_stepper_dependencies(int nx, int ny, int bc_x, int bc_y, int tx, int ty, int* off, int off_cap, int* idx,
                            int idx_cap, int* nnz) {
    if (nx <= 0 || ny <= 0 || tx <= 0 || ty <= 0 || !nnz) return set_error(FV_ERR_ARG, "fv_stepper_dependencies: bad arguments");
    if (!valid_common(FLUX_HLLC, LIM_NONE, bc_x, bc_y)) return set_error(FV_ERR_ARG, "fv_stepper_dependencies: unknown bc");
    std::vector<int> o, ix;
    build_stepper_deps(nx, ny, bc_x, bc_y, tx, ty, o, ix);
    *nnz = (int)ix.size();
    if (off && off_cap >= (int)o.size()) std::memcpy(off, o.data(), o.size() * sizeof(int));
    if (idx && idx_cap >= (int)ix.size()) std::memcpy(idx, ix.data(), ix.size() * sizeof(int));
    return FV_OK;
}

int fv_autotune(fv_solver* s, int steps, int* variant) {
    if (!s) return set_error(FV_ERR_ARG, "fv_autotune: NULL handle");
    if (!s->has_state) return set_error(FV_ERR_STATE, "fv_autotune: no state set");
    int v = 0;
    int rc = autotune(s, steps > 0 ? steps : 8, &v);
    if (rc == FV_OK && variant) *variant = v;
    return rc;
}

int fv_set_tile(fv_solver* s, int variant) {
    if (!s) return set_error(FV_ERR_ARG, "fv_set_tile: NULL handle");
    if (variant < 0 || variant >= (int)variants().size()) return set_error(FV_ERR_ARG, "fv_set_tile: no variant %d", variant);
    s->variant = variant;
    s->tuned = true;
    return FV_OK;
}

int fv_get_tile(fv_solver* s, int* variant) {
    if (!s || !variant) return set_error(FV_ERR_ARG, "fv_get_tile: NULL argument");
    *variant = s->variant;
    return FV_OK;
}

int fv_tile_variant(int variant, int* tx, int* ty, int* threads) {
    if (variant < 0 || variant >= (int)variants().size()) return set_error(FV_ERR_ARG, "fv_tile_variant: no variant %d", variant);
    const TileVariant& v = variants()[variant];
    if (tx) *tx = v.tx;
    if (ty) *ty = v.ty;
    if (threads) *threads = v.nt;
    return FV_OK;
}

int fv_profile(fv_solver* s, int enable) {
    if (!s) return set_error(FV_ERR_ARG, "fv_profile: NULL handle");
    if (enable && !s->ev[0][0]) {
        for (auto& tri : s->ev)
            for (cudaEvent_t& e : tri) FV_CUDA(cudaEventCreate(&e));
        for (cudaEvent_t& e : s->sev) FV_CUDA(cudaEventCreate(&e));
    }
    while (s->ring_used) {
        int rc = retire_oldest(s);
        if (rc) return rc;
    }
    s->profiling = enable != 0;
    s->ms1 = s->ms2 = 0.0;
    s->timed = 0;
    s->step_ms = 0.0;
    s->step_steps = s->step_launches = 0;
    return FV_OK;
}

int fv_profile_steps(fv_solver* s, double* ms_per_step, long long* steps, long long* launches) {
    if (!s) return set_error(FV_ERR_ARG, "fv_profile_steps: NULL handle");
    while (s->ring_used) {
        int rc = retire_oldest(s);
        if (rc) return rc;
    }
    const long long n = s->step_steps + s->timed;
    const double ms = s->step_ms + s->ms1 + s->ms2;  // ms1, ms2: totals over the timed per-stage steps
    if (ms_per_step) *ms_per_step = n ? ms / n : 0.0;
    if (steps) *steps = n;
    if (launches) *launches = s->step_launches;
    return FV_OK;
}

int fv_stepper_launch(fv_solver* s, int* variant, int* ctas_per_sm, int* ctas) {
    if (!s) return set_error(FV_ERR_ARG, "fv_stepper_launch: NULL handle");
    const bool on = stepper_enabled() && s->svariant >= 0 && s->sgrid > 0;
    int sms = 1;
    if (on) FV_CUDA(cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, s->device));
    if (variant) *variant = on ? s->svariant : -1;
    if (ctas_per_sm) *ctas_per_sm = on ? s->sgrid / sms : 0;
    if (ctas) *ctas = on ? s->sgrid : 0;
    return FV_OK;
}

int fv_stepper_tile(fv_solver* s, int* tx, int* ty, int* threads) {
    if (!s) return set_error(FV_ERR_ARG, "fv_stepper_tile: NULL handle");
    if (!stepper_enabled() || s->svariant < 0) {
        if (tx) *tx = 0;
        if (ty) *ty = 0;
        if (threads) *threads = 0;
        return FV_OK;
    }
    const StepperVariant& v = stepper_variants()[s->svariant];
    if (tx) *tx = v.tx;
    if (ty) *ty = v.ty;
    if (threads) *threads = v.nt;
    return FV_OK;
}

int fv_profile_read(fv_solver* s, double* ms1, double* ms2, long long* steps) {
    if (!s) return set_error(FV_ERR_ARG, "fv_profile_read: NULL handle");
    while (s->ring_used) {
        int rc = retire_oldest(s);
        if (rc) return rc;
    }
    if (ms1) *ms1 = s->timed ? s->ms1 / s->timed : 0.0;
    if (ms2) *ms2 = s->timed ? s->ms2 / s->timed : 0.0;
    if (steps) *steps = s->timed;
    return FV_OK;
}

int fv_launch_count(fv_solver* s, long long* n) {
    if (!s || !n) return set_error(FV_ERR_ARG, "fv_launch_count: NULL argument");
    *n = s->launches;
    return FV_OK;
}

int fv_synchronize(fv_solver* s) {
    if (!s) return set_error(FV_ERR_ARG, "fv_synchronize: NULL handle");
    FV_CUDA(cudaStreamSynchronize(s->stream));
    return FV_OK;
}

int fv_get_stream(fv_solver* s, void** stream) {
    if (!s || !stream) return set_error(FV_ERR_ARG, "fv_get_stream: NULL argument");
    *stream = static_cast<void*>(s->stream);
    return FV_OK;
}

}  // extern "C"
