// fv_step_noalloc: one SSP-RK2 step on a caller-owned device state that allocates no device memory.
//
// Some callers cannot call cudaMalloc when they want to step: a host that runs inside another
// framework's memory pool (a training process whose allocator has reserved the GPU's memory, where a
// raw cudaMalloc would fail or fragment the pool), or a real-time driver loop that forbids allocation
// after start-up.  fv_create allocates the state and scratch of a handle up front, which such a
// caller cannot do at that point.  This entry point takes the state as a device pointer and keeps its
// scratch (the intermediate RK stage U1, the primitives W and W1 and the control block) in the
// file-scope array below, which every GPU that loads this library holds until the process exits.
//
// Limits and sharing: grids of at most FV_NOALLOC_MAX_CELLS cells; larger ones are rejected with
// FV_ERR_ARG.  All calls on a device share the one scratch array, and it keeps the last call's
// contents, so calls whose work overlaps on the GPU (other streams, other host threads) race and
// must be serialised by the caller.  The control block is cleared at the start of every call.
// The first call on a device (that device current) looks up the array's device address with
// cudaGetSymbolAddress and sets the kernels' shared-memory limit; make that first call before any
// stream capture.  That set-up is cached for the life of the process: after cudaDeviceReset the
// library's module may be reloaded at another address, so do not use this entry point across a
// device reset.
// The kernels move each cell with two 16-byte (double2) accesses, so d_U must be 16-byte aligned
// (cudaMalloc'd memory is; a view at an odd double offset is not): a misaligned pointer is rejected
// with FV_ERR_ARG before anything is launched.
#include <cuda_runtime.h>

#include <algorithm>
#include <climits>
#include <cstdint>
#include <mutex>

#include "../../include/fv.h"
#include "fv_kernels.cuh"

int fv_internal_set_error(int code, const char* msg);  // fv_api.cu: sets fv_last_error()

using namespace fv;

namespace {

constexpr size_t kStateBytes = size_t(FV_NOALLOC_MAX_CELLS) * sizeof(Q4);
// layout: U1 | W | W1 | control block
constexpr size_t kScratchBytes = 3 * kStateBytes + ((sizeof(FvCtrl) + 255) / 256) * 256;

static __device__ __align__(256) unsigned char g_noalloc_scratch[kScratchBytes];

// Tile shape of the stage kernels used here (the handle API's default shape; no autotuning, which
// would need buffers of its own).
constexpr int TX = 32, TY = 8, NT = 256, MINB = 4;

constexpr int kMaxDevices = 64;
std::mutex g_mu;
unsigned char* g_dev_ptr[kMaxDevices] = {};

using StageFn = void (*)(GridDesc, TileMaps);

template <int F, int L>
void pick(StageFn* s1, StageFn* s2) {
    *s1 = stage_kernel<F, L, 1, TX, TY, NT, MINB>;
    *s2 = stage_kernel<F, L, 2, TX, TY, NT, MINB>;
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

// Once per device, with that device current: the device address of the scratch array (in host code
// g_noalloc_scratch names a host-side stand-in, never a device address) and the stage kernels'
// dynamic shared-memory limit.
int setup(int dev, unsigned char** out) {
    std::lock_guard<std::mutex> lock(g_mu);
    if (!g_dev_ptr[dev]) {
        void* p = nullptr;
        cudaError_t e = cudaGetSymbolAddress(&p, g_noalloc_scratch);
        if (e != cudaSuccess || !p) return fv_internal_set_error(FV_ERR_CUDA, cudaGetErrorString(e));
        for (int f = 0; f < 2; ++f)
            for (int l = 0; l < 4; ++l) {
                StageFn s1, s2;
                stage_pair(f, l, &s1, &s2);
                for (StageFn k : {s1, s2}) {
                    e = cudaFuncSetAttribute((const void*)k, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                             (int)sizeof(TileSmem<TX, TY>));
                    if (e != cudaSuccess) return fv_internal_set_error(FV_ERR_CUDA, cudaGetErrorString(e));
                }
            }
        g_dev_ptr[dev] = static_cast<unsigned char*>(p);
    }
    *out = g_dev_ptr[dev];
    return FV_OK;
}

}  // namespace

extern "C" int fv_step_noalloc(int nx, int ny, double x_min, double x_max, double y_min, double y_max, int bc_x,
                               int bc_y, int flux, int limiter, double* d_U, double dt, void* stream) {
    if (!d_U) return fv_internal_set_error(FV_ERR_ARG, "fv_step_noalloc: d_U is NULL");
    if (reinterpret_cast<uintptr_t>(d_U) & 15u)
        return fv_internal_set_error(FV_ERR_ARG, "fv_step_noalloc: d_U must be 16-byte aligned");
    if (nx <= 0 || ny <= 0) return fv_internal_set_error(FV_ERR_ARG, "fv_step_noalloc: nx and ny must be positive");
    if ((long long)nx * ny > FV_NOALLOC_MAX_CELLS)
        return fv_internal_set_error(FV_ERR_ARG,
                                     "fv_step_noalloc: grid larger than FV_NOALLOC_MAX_CELLS (16384 cells); "
                                     "use fv_create/fv_step for larger grids");
    if (!(x_max > x_min) || !(y_max > y_min)) return fv_internal_set_error(FV_ERR_ARG, "fv_step_noalloc: empty domain");
    if ((flux != FLUX_HLLC && flux != FLUX_RUSANOV) || limiter < LIM_NONE || limiter > LIM_VANLEER ||
        (bc_x != BC_PERIODIC && bc_x != BC_TRANSMISSIVE) || (bc_y != BC_PERIODIC && bc_y != BC_TRANSMISSIVE))
        return fv_internal_set_error(FV_ERR_ARG, "fv_step_noalloc: unknown flux/limiter/bc id");
    int dev = 0;
    if (cudaGetDevice(&dev) != cudaSuccess || dev < 0 || dev >= kMaxDevices)
        return fv_internal_set_error(FV_ERR_CUDA, "fv_step_noalloc: no usable CUDA device");
    unsigned char* base = nullptr;
    int rc = setup(dev, &base);
    if (rc) return rc;

    GridDesc g{};
    g.U = reinterpret_cast<Q4*>(d_U);
    g.U1 = reinterpret_cast<Q4*>(base);
    g.W = reinterpret_cast<Q4*>(base + kStateBytes);
    g.W1 = reinterpret_cast<Q4*>(base + 2 * kStateBytes);
    g.ctrl = reinterpret_cast<FvCtrl*>(base + 3 * kStateBytes);
    g.nx = nx; g.ny = ny; g.bc_x = bc_x; g.bc_y = bc_y;
    g.dx = (x_max - x_min) / nx;  // make_grid, grid2d.hpp:34-35
    g.dy = (y_max - y_min) / ny;
    g.cfl = 0.5;                   // unused by a fixed-dt step
    g.cx = 1.0 / g.dx;
    g.cy = 1.0 / g.dy;
    cudaStream_t st = static_cast<cudaStream_t>(stream);
    const int n = nx * ny;
    StageFn s1, s2;
    stage_pair(flux, limiter, &s1, &s2);
    const dim3 grid((nx + TX - 1) / TX, (ny + TY - 1) / TY);
    // clear the control block (the array keeps the previous call's contents), fixed-dt mode, W = prim(U)
    ctrl_reset_kernel<<<1, 1, 0, st>>>(g.ctrl, 0.0, 1);
    ctrl_set_kernel<<<1, 1, 0, st>>>(g.ctrl, MODE_FIXED, 0.0, dt);
    wave_speed_kernel<<<std::max(1, std::min((n + RED_NT - 1) / RED_NT, 148 * 8)), RED_NT, 0, st>>>(g.U, g.W, n, g.ctrl);
    const TileMaps no_tma{};  // every tile loads through the BC index map
    s1<<<grid, NT, sizeof(TileSmem<TX, TY>), st>>>(g, no_tma);
    s2<<<grid, NT, sizeof(TileSmem<TX, TY>), st>>>(g, no_tma);
    const cudaError_t e = cudaGetLastError();
    if (e != cudaSuccess) return fv_internal_set_error(FV_ERR_CUDA, cudaGetErrorString(e));
    return FV_OK;
}
