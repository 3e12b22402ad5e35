// Harness around the reference solver core (TEST INFRASTRUCTURE ONLY).
//
// Compiled by oracle/build_oracle.py against the reference's own headers where they lie
// (solver/src/{state2d,grid2d,limiters,riemann2d,solver2d,riemann,state}.hpp of
// GusGus2004/neural-pde-surrogate); nothing from the reference is copied here.  The output goes to
// oracle/_ref/libfvref.so, which the tests use to pin the C restatement in oracle/fv_oracle.c and
// which bench.py may time as the CPU reference arm.
//
// Only the pieces of the reference that need HDF5 cannot be compiled here (main2d.cpp, io_hdf5.hpp,
// trajectory.hpp).  Their two non-I/O algorithms are restated below, following the cited lines:
// the frame time loop (main2d.cpp:224-246) and TrajectoryWriter::add (trajectory.hpp:31-51).
#include "solver2d.hpp"
#include "riemann.hpp"   // 1D flux, the comparison used by the reference's test_riemann2d.cpp

#ifdef _OPENMP
#include <omp.h>
#endif
#include <memory>
#include <vector>

namespace {

struct RefRun {
    e2d::Grid g;
    std::unique_ptr<e2d::Solver> solver;
    std::vector<e2d::Conserved> U;
};

e2d::FluxFn pick_flux(int id) { return id == 1 ? e2d::hllc_flux : e2d::rusanov_flux; }
Limiter pick_lim(int id) {
    switch (id) {
    case 0: return no_slope;
    case 1: return unlimited;
    case 2: return minmod;
    default: return van_leer;
    }
}

// The reference's compute_dt exits the process on a non-physical cell; check first so the harness
// can return an error instead.  Same predicate as solver2d.hpp:75.
bool first_bad(const RefRun& r, int* bi, int* bj, double* brho, double* bp) {
    for (int j = 0; j < r.g.ny; ++j)
        for (int i = 0; i < r.g.nx; ++i) {
            e2d::Primitive W = e2d::to_primitive(r.U[r.g.idx(i, j)]);
            if (!(W.rho > 0.0) || !(W.p > 0.0)) {
                if (bi) *bi = i;
                if (bj) *bj = j;
                if (brho) *brho = W.rho;
                if (bp) *bp = W.p;
                return true;
            }
        }
    return false;
}

}  // namespace

extern "C" {

// one cell between the harness's flat (rho, rho*u, rho*v, E) doubles and the reference's Conserved
static e2d::Conserved load_c(const double* p) { return e2d::Conserved{p[0], p[1], p[2], p[3]}; }
static void store_c(double* p, const e2d::Conserved& c) { p[0] = c.rho; p[1] = c.mx; p[2] = c.my; p[3] = c.E; }

void* ref_create(int nx, int ny, double x_min, double x_max, double y_min, double y_max, int bc_x, int bc_y,
                 int flux, int lim, double cfl) {
    auto* r = new RefRun;
    r->g = e2d::make_grid(nx, ny, x_min, x_max, y_min, y_max, bc_x ? e2d::BC::Periodic : e2d::BC::Transmissive,
                          bc_y ? e2d::BC::Periodic : e2d::BC::Transmissive);
    r->solver = std::make_unique<e2d::Solver>(r->g, pick_flux(flux), pick_lim(lim), cfl);
    r->U.assign(r->g.size(), e2d::Conserved{});
    return r;
}

void ref_destroy(void* h) { delete static_cast<RefRun*>(h); }

void ref_set_state(void* h, const double* U) {
    auto* r = static_cast<RefRun*>(h);
    for (int j = 0; j < r->g.ny; ++j)
        for (int i = 0; i < r->g.nx; ++i)
            r->U[r->g.idx(i, j)] = load_c(U + (size_t(j) * r->g.nx + i) * 4);
}

void ref_get_state(void* h, double* U) {
    auto* r = static_cast<RefRun*>(h);
    for (int j = 0; j < r->g.ny; ++j)
        for (int i = 0; i < r->g.nx; ++i)
            store_c(U + (size_t(j) * r->g.nx + i) * 4, r->U[r->g.idx(i, j)]);
}

int ref_compute_dt(void* h, double* dt, int* bi, int* bj, double* brho, double* bp) {
    auto* r = static_cast<RefRun*>(h);
    if (first_bad(*r, bi, bj, brho, bp)) return 1;
    *dt = r->solver->compute_dt(r->U);
    return 0;
}

void ref_step(void* h, double dt) {
    auto* r = static_cast<RefRun*>(h);
    r->solver->step(r->U, dt);
}

// main2d.cpp:237-242
int ref_advance_to(void* h, double t_next, double* t, long long* steps, int* bi, int* bj, double* brho, double* bp) {
    auto* r = static_cast<RefRun*>(h);
    while (*t < t_next) {
        if (first_bad(*r, bi, bj, brho, bp)) return 1;
        double dt = std::min(r->solver->compute_dt(r->U), t_next - *t);
        r->solver->step(r->U, dt);
        *t += dt;
        ++*steps;
    }
    return 0;
}

// trajectory.hpp:31-51 for one level
void ref_block_average(void* h, int f, float* out) {
    auto* r = static_cast<RefRun*>(h);
    const e2d::Grid& g = r->g;
    const int nxc = g.nx / f, nyc = g.ny / f;
    const double inv = 1.0 / (double(f) * f);
    for (int jc = 0; jc < nyc; ++jc)
        for (int ic = 0; ic < nxc; ++ic) {
            double s[4] = {0.0, 0.0, 0.0, 0.0};
            for (int j = jc * f; j < (jc + 1) * f; ++j)
                for (int i = ic * f; i < (ic + 1) * f; ++i) {
                    const e2d::Conserved& c = r->U[g.idx(i, j)];
                    s[0] += c.rho; s[1] += c.mx; s[2] += c.my; s[3] += c.E;
                }
            for (int q = 0; q < 4; ++q) out[(size_t(q) * nyc + jc) * nxc + ic] = float(s[q] * inv);
        }
}

void ref_apply_bcs_ghosted(int nx, int ny, int bc_x, int bc_y, double* Ug) {
    e2d::Grid g = e2d::make_grid(nx, ny, 0.0, 1.0, 0.0, 1.0, bc_x ? e2d::BC::Periodic : e2d::BC::Transmissive,
                                 bc_y ? e2d::BC::Periodic : e2d::BC::Transmissive);
    std::vector<e2d::Conserved> U(g.size());
    for (size_t k = 0; k < U.size(); ++k) U[k] = load_c(Ug + 4 * k);
    e2d::apply_bcs(g, U);
    for (size_t k = 0; k < U.size(); ++k) store_c(Ug + 4 * k, U[k]);
}

void ref_flux(int flux, const double* UL, const double* UR, double* F) {
    store_c(F, pick_flux(flux)(load_c(UL), load_c(UR)));
}

void ref_flux_y(int flux, const double* UL, const double* UR, double* F) {
    store_c(F, e2d::flux_y_face(pick_flux(flux), load_c(UL), load_c(UR)));
}

void ref_hllc_1d(const double* UL, const double* UR, double* F) {
    Conserved a{UL[0], UL[1], UL[2]}, b{UR[0], UR[1], UR[2]};
    Conserved c = hllc_flux(a, b);
    F[0] = c.rho; F[1] = c.mom; F[2] = c.E;
}

int ref_max_threads() {
#ifdef _OPENMP
    return omp_get_max_threads();
#else
    return 1;
#endif
}

}  // extern "C"
