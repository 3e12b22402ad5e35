// C-ABI of the finite-volume solver (include/fv.h): handle management, host<->device copies, the
// device-resident time loop, trajectory output.  No torch types, no exits, no CPU fallback: every
// compute call launches the sm_100a kernels of fv_kernels.cuh.
#include <cuda_runtime.h>

#include <algorithm>
#include <cmath>
#include <cstdarg>
#include <cstdio>
#include <cstring>
#include <string>
#include <vector>

#include "../../include/fv.h"
#include "fv_kernels.cuh"

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

using StageFn = void (*)(StageArgs);

template <int F, int L>
void pick_stage(StageFn* s1, StageFn* s2) {
    *s1 = stage_kernel<F, L, 1>;
    *s2 = stage_kernel<F, L, 2>;
}

void stage_fns(int flux, int lim, StageFn* s1, StageFn* s2) {
    if (flux == FLUX_HLLC) {
        switch (lim) {
        case LIM_NONE: pick_stage<FLUX_HLLC, LIM_NONE>(s1, s2); break;
        case LIM_UNLIMITED: pick_stage<FLUX_HLLC, LIM_UNLIMITED>(s1, s2); break;
        case LIM_MINMOD: pick_stage<FLUX_HLLC, LIM_MINMOD>(s1, s2); break;
        default: pick_stage<FLUX_HLLC, LIM_VANLEER>(s1, s2); break;
        }
    } else {
        switch (lim) {
        case LIM_NONE: pick_stage<FLUX_RUSANOV, LIM_NONE>(s1, s2); break;
        case LIM_UNLIMITED: pick_stage<FLUX_RUSANOV, LIM_UNLIMITED>(s1, s2); break;
        case LIM_MINMOD: pick_stage<FLUX_RUSANOV, LIM_MINMOD>(s1, s2); break;
        default: pick_stage<FLUX_RUSANOV, LIM_VANLEER>(s1, s2); break;
        }
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
    FvCtrl* ctrl = nullptr;
    FvCtrl* h_ctrl = nullptr;  // pinned mirror
    int* d_count = nullptr;
    int* h_count = nullptr;
    double* d_prim = nullptr;  // staging for fv_set_primitive (4 * n doubles), allocated on first use
    float* d_avg = nullptr;
    size_t d_avg_cap = 0;
    StageFn s1 = nullptr, s2 = nullptr;
    dim3 grid;
    bool has_state = false;
    long long launches = 0;  // kernels launched by this handle
    // kernel timing (fv_profile): a ring of event triples bracketing stage 1 and stage 2
    static constexpr int kRing = 256;
    bool profiling = false;
    cudaEvent_t ev[kRing][3] = {};
    int ring_head = 0, ring_used = 0;
    double ms1 = 0.0, ms2 = 0.0;
    long long timed = 0;

    size_t ncell() const { return size_t(nx) * ny; }
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

int launch_step(fv_solver* s) {
    StageArgs a1{};
    a1.Uin = s->U; a1.Ubase = s->U; a1.Uout = s->U1;
    a1.nx = s->nx; a1.ny = s->ny; a1.bc_x = s->bc_x; a1.bc_y = s->bc_y;
    a1.cx = 1.0 / s->dx; a1.cy = 1.0 / s->dy; a1.dx = s->dx; a1.dy = s->dy; a1.cfl = s->cfl;
    a1.ctrl = s->ctrl;
    StageArgs a2 = a1;
    a2.Uin = s->U1; a2.Ubase = s->U; a2.Uout = s->U;
    cudaEvent_t* ev = nullptr;
    if (s->profiling) {
        if (s->ring_used == fv_solver::kRing) {  // retire the oldest triple before reusing it
            int rc = retire_oldest(s);
            if (rc) return rc;
        }
        ev = s->ev[(s->ring_head + s->ring_used) % fv_solver::kRing];
        s->ring_used++;
        FV_CUDA(cudaEventRecord(ev[0], s->stream));
    }
    s->s1<<<s->grid, NT, sizeof(StageSmem), s->stream>>>(a1);
    if (ev) FV_CUDA(cudaEventRecord(ev[1], s->stream));
    s->s2<<<s->grid, NT, sizeof(StageSmem), s->stream>>>(a2);
    if (ev) FV_CUDA(cudaEventRecord(ev[2], s->stream));
    s->launches += 2;
    FV_CUDA(cudaGetLastError());
    return FV_OK;
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
    const int blocks = std::max(1, std::min((n + NT - 1) / NT, 148 * 8));
    wave_speed_kernel<<<blocks, NT, 0, s->stream>>>(s->U, n, s->ctrl);
    s->launches += 2;
    FV_CUDA(cudaGetLastError());
    s->has_state = true;
    return FV_OK;
}

bool valid_common(int flux, int lim, int bc_x, int bc_y) {
    return (flux == FLUX_HLLC || flux == FLUX_RUSANOV) && lim >= LIM_NONE && lim <= LIM_VANLEER &&
           (bc_x == BC_PERIODIC || bc_x == BC_TRANSMISSIVE) && (bc_y == BC_PERIODIC || bc_y == BC_TRANSMISSIVE);
}

}  // namespace

extern "C" {

const char* fv_last_error(void) { return g_last_error.c_str(); }
const char* fv_version(void) { return "fv-b200 1.0 (sm_100a, FP64, bit-exact build)"; }

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
    stage_fns(flux, limiter, &s->s1, &s->s2);
    s->grid = dim3((nx + TX - 1) / TX, (ny + TY - 1) / TY);
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
    if (rc == FV_OK && (e = cudaMalloc(&s->ctrl, sizeof(FvCtrl))) != cudaSuccess) fail(e, "control block");
    if (rc == FV_OK && (e = cudaMalloc(&s->d_count, sizeof(int))) != cudaSuccess) fail(e, "counter");
    if (rc == FV_OK && (e = cudaMallocHost(&s->h_ctrl, sizeof(FvCtrl))) != cudaSuccess) fail(e, "pinned control");
    if (rc == FV_OK && (e = cudaMallocHost(&s->h_count, sizeof(int))) != cudaSuccess) fail(e, "pinned counter");
    if (rc == FV_OK && (e = cudaMemsetAsync(s->ctrl, 0, sizeof(FvCtrl), s->stream)) != cudaSuccess) fail(e, "memset");
    if (rc == FV_OK) {
        for (StageFn f : {s->s1, s->s2}) {
            if ((e = cudaFuncSetAttribute((const void*)f, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                          (int)sizeof(StageSmem))) != cudaSuccess) {
                fail(e, "smem attribute");
                break;
            }
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
    cudaFree(s->U);
    cudaFree(s->U1);
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
    // Steps are queued in batches sized from the last dt; steps queued after t reaches t_next (or
    // after a non-physical state) exit at their first instruction, so a batch may overshoot freely.
    const int kMaxBatch = 256;
    for (;;) {
        const FvCtrl& c = *s->h_ctrl;
        if (c.status) break;
        const double t = c.t[c.step & 1];
        if (!(t < t_next)) break;
        double dt_est = c.dt;
        if (!(dt_est > 0.0)) {
            double sx, sy;
            std::memcpy(&sx, &c.sxy[c.step & 1][0], 8);
            std::memcpy(&sy, &c.sxy[c.step & 1][1], 8);
            dt_est = s->cfl / (sx / s->dx + sy / s->dy);
        }
        double est = (dt_est > 0.0) ? std::ceil((t_next - t) / dt_est) : 1.0;
        int batch = (int)std::min<double>(std::max(est, 1.0) + 1.0, (double)kMaxBatch);
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

int fv_profile(fv_solver* s, int enable) {
    if (!s) return set_error(FV_ERR_ARG, "fv_profile: NULL handle");
    if (enable && !s->ev[0][0]) {
        for (auto& tri : s->ev)
            for (cudaEvent_t& e : tri) FV_CUDA(cudaEventCreate(&e));
    }
    while (s->ring_used) {
        int rc = retire_oldest(s);
        if (rc) return rc;
    }
    s->profiling = enable != 0;
    s->ms1 = s->ms2 = 0.0;
    s->timed = 0;
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

}  // extern "C"
