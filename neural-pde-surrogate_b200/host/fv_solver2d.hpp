// Drop-in for the reference's e2d::Solver (solver/src/solver2d.hpp:53-113) over libfv's C-ABI
// (include/fv.h): the same constructor, compute_dt, step and profile, so the reference's C++ callers
// build against the GPU solver by including this header where they included solver2d.hpp.
//
// It needs the reference's own grid2d.hpp, riemann2d.hpp and limiters.hpp on the include path: their
// Grid, Conserved, FluxFn and Limiter are this class's argument types, and the addresses of their
// flux and limiter functions select the GPU kernels (hllc_flux / rusanov_flux; no_slope, unlimited,
// minmod, van_leer).  Any other function pointer is rejected with std::invalid_argument.
//
// Per call, on the caller's ghosted std::vector<Conserved> (grid2d.hpp:12-28):
//  * compute_dt(U): the CFL dt of U's physical cells, bit-identical to the reference's
//    (solver2d.hpp:67-83).  A non-physical cell prints the reference's message for the first bad cell
//    in row-major order and exits with status 1, as report_bad_cell does (solver2d.hpp:116-126).
//  * step(U, dt): fills U's ghost cells with the reference's apply_bcs, as the first compute_rhs of
//    its step does (solver2d.hpp:129-131), then runs one SSP-RK2 step on the GPU and copies the
//    physical cells back: U ends bit-identical to the reference's, ghost cells included.
// The physical cells cross PCIe only when they changed: the last state sent or fetched stays on the
// host and is compared byte for byte.  A compute_dt/step loop therefore moves one state per step (the
// fetch after the step); fv_advance_to, which keeps the whole loop on the GPU, moves none.
//
// Profile keeps host wall time per call kind; print(steps, cells) has the reference's layout
// (solver2d.hpp:29-52) with this solver's phases.
#pragma once
#include "grid2d.hpp"
#include "limiters.hpp"
#include "riemann2d.hpp"

#include "fv.h"

#include <array>
#include <chrono>
#include <cstdio>
#include <cstdlib>
#include <cstring>
#include <iostream>
#include <stdexcept>
#include <vector>

namespace e2d {

static_assert(sizeof(Conserved) == 4 * sizeof(double), "Conserved must be four packed doubles (fv.h AoS layout)");

struct Profile {
    enum Phase { DT, STEP, COPY, N_PHASES };
    static constexpr const char* names[N_PHASES] = {"compute_dt (GPU, wave speeds)", "step (GPU, SSP-RK2)",
                                                    "host <-> device state copies"};
    std::array<double, N_PHASES> secs{};

    void print(long steps, long cells) const {
        double total = 0.0;
        for (double x : secs) total += x;
        std::printf("\n%-30s %9s %7s %12s\n", "phase", "time (s)", "share", "ns per cell");
        for (int k = 0; k < N_PHASES; ++k)
            std::printf("%-30s %9.3f %6.1f%% %12.2f\n", names[k], secs[k], total > 0 ? 100.0 * secs[k] / total : 0.0,
                        1e9 * secs[k] / (double(steps) * cells));
        std::printf("%-30s %9.3f %6.1f%% %12.2f\n", "total", total, 100.0, 1e9 * total / (double(steps) * cells));
    }
};

class Solver {
public:
    Solver(const Grid& grid, FluxFn flux, Limiter lim, double cfl)
        : g(grid), shadow(size_t(grid.nx) * grid.ny), packed(size_t(grid.nx) * grid.ny) {
        if (fv_create(g.nx, g.ny, g.x_min, g.x_max, g.y_min, g.y_max, bc_id(g.bc_x), bc_id(g.bc_y), flux_id(flux),
                      limiter_id(lim), cfl, nullptr, &h) != FV_OK)
            throw std::runtime_error(fv_last_error());
    }
    ~Solver() { fv_destroy(h); }
    Solver(const Solver&) = delete;
    Solver& operator=(const Solver&) = delete;

    const Profile& profile() const { return prof; }

    double compute_dt(const std::vector<Conserved>& U) const {
        send(U);
        const auto t0 = clock::now();
        double dt = 0.0;
        fv_bad_cell bad{};
        const int rc = fv_compute_dt(h, &dt, &bad);
        prof.secs[Profile::DT] += seconds(t0);
        if (rc == FV_ERR_NONPHYSICAL) {
            std::cerr << "Non-physical state in cell (" << bad.i << ", " << bad.j << "): rho = " << bad.rho
                      << ", p = " << bad.p << '\n';
            std::exit(1);
        }
        check(rc);
        return dt;
    }

    void step(std::vector<Conserved>& U, double dt) {
        apply_bcs(g, U);
        send(U);
        auto t0 = clock::now();
        check(fv_step(h, dt));
        check(fv_get_state(h, reinterpret_cast<double*>(shadow.data())));  // waits for the step
        prof.secs[Profile::STEP] += seconds(t0);
        t0 = clock::now();
        for (int j = 0; j < g.ny; ++j)
            std::memcpy(&U[g.idx(0, j)], &shadow[size_t(j) * g.nx], size_t(g.nx) * sizeof(Conserved));
        prof.secs[Profile::COPY] += seconds(t0);
    }

private:
    using clock = std::chrono::steady_clock;
    Grid g;
    fv_solver* h = nullptr;
    mutable std::vector<Conserved> shadow;  // the physical cells the GPU holds
    mutable std::vector<Conserved> packed;  // the caller's physical cells, rows packed
    mutable bool synced = false;
    mutable Profile prof;

    static double seconds(clock::time_point t0) { return std::chrono::duration<double>(clock::now() - t0).count(); }

    static void check(int rc) {
        if (rc != FV_OK) throw std::runtime_error(fv_last_error());
    }

    // Sends U's physical cells unless the GPU already holds exactly these bytes.
    void send(const std::vector<Conserved>& U) const {
        const auto t0 = clock::now();
        for (int j = 0; j < g.ny; ++j)
            std::memcpy(&packed[size_t(j) * g.nx], &U[g.idx(0, j)], size_t(g.nx) * sizeof(Conserved));
        if (!synced || std::memcmp(packed.data(), shadow.data(), packed.size() * sizeof(Conserved)) != 0) {
            check(fv_set_state(h, reinterpret_cast<const double*>(packed.data())));
            shadow.swap(packed);
            synced = true;
        }
        prof.secs[Profile::COPY] += seconds(t0);
    }

    static int bc_id(BC bc) { return bc == BC::Periodic ? FV_BC_PERIODIC : FV_BC_TRANSMISSIVE; }

    static int flux_id(FluxFn f) {
        if (f == &hllc_flux) return FV_FLUX_HLLC;
        if (f == &rusanov_flux) return FV_FLUX_RUSANOV;
        throw std::invalid_argument("Solver: the flux must be hllc_flux or rusanov_flux");
    }

    static int limiter_id(Limiter l) {
        if (l == &no_slope) return FV_LIM_NONE;
        if (l == &unlimited) return FV_LIM_UNLIMITED;
        if (l == &minmod) return FV_LIM_MINMOD;
        if (l == &van_leer) return FV_LIM_VANLEER;
        throw std::invalid_argument("Solver: the limiter must be no_slope, unlimited, minmod or van_leer");
    }
};

}  // namespace e2d
