// euler2d: the reference's 2D Euler driver (solver/src/main2d.cpp) over the B200 C-ABI (include/fv.h).
//
//   euler2d --test lax_liu3 --n 256 --scheme hllc --limiter vanleer --nout 10 --out runs
//   euler2d --init ic.npz --nout 50 --tstart 0.1 --traj traj.npz --save 128,64
//
// Same options, defaults, test problems, time loop and messages as main2d.cpp:25-262.  The loop
// `dt = min(compute_dt(U), t_next - t); step; t += dt` (main2d.cpp:224-246) runs on the GPU inside
// fv_advance_to / fv_run_trajectory, with bit-identical times, step counts and states.
//
// Files: libhdf5 is not available to this build, so snapshots, initial conditions and trajectories
// are .npz archives holding the reference's HDF5 datasets and attributes under the same names and
// shapes (io_hdf5.hpp:56-97, :170-206; trajectory.hpp:53-91); numpy.load() reads them.
#include <chrono>
#include <cmath>
#include <cstdio>
#include <cstdlib>
#include <filesystem>
#include <iostream>
#include <map>
#include <memory>
#include <string>
#include <vector>

#include "../../include/fv.h"
#include "npz_io.hpp"

namespace {

constexpr double GAMMA = 1.4;  // state2d.hpp:7

std::map<std::string, std::string> parse_args(int argc, char* argv[]) {
    std::map<std::string, std::string> a = {
        {"test", "lax_liu3"}, {"n", "256"}, {"scheme", "hllc"}, {"limiter", "vanleer"}, {"cfl", "0.5"},
        {"nout", "10"}, {"out", "runs"}, {"tend", "default"}, {"profile", "no"}, {"init", ""}, {"traj", ""},
        {"save", ""}, {"tstart", "0"}};
    for (int k = 1; k < argc; ++k) {
        std::string key = argv[k];
        if (key.rfind("--", 0) != 0 || k + 1 >= argc) {
            std::cerr << "Expected '--key value', got '" << key << "'\n";
            std::exit(1);
        }
        key = key.substr(2);
        if (!a.count(key)) {
            std::cerr << "Unknown option --" << key << '\n';
            std::exit(1);
        }
        a[key] = argv[++k];
    }
    return a;
}

std::vector<int> parse_sizes(const std::string& s) {  // trajectory.hpp:104-114
    std::vector<int> out;
    size_t start = 0;
    while (start < s.size()) {
        size_t end = s.find(',', start);
        if (end == std::string::npos) end = s.size();
        out.push_back(std::stoi(s.substr(start, end - start)));
        start = end + 1;
    }
    return out;
}

struct Problem {
    int nx = 0, ny = 0;
    double x_min = 0, x_max = 1, y_min = 0, y_max = 1;
    int bc_x = FV_BC_TRANSMISSIVE, bc_y = FV_BC_TRANSMISSIVE;
    double t_end = 0.0;
    std::vector<double> rho, u, v, p;  // primitive initial state, row-major (ny, nx)

    double dx() const { return (x_max - x_min) / nx; }
    double dy() const { return (y_max - y_min) / ny; }
    double xc(int i) const { return x_min + (i + 0.5) * dx(); }  // grid2d.hpp:26-27
    double yc(int j) const { return y_min + (j + 0.5) * dy(); }
    void alloc() {
        const size_t n = size_t(nx) * ny;
        rho.assign(n, 0.0); u.assign(n, 0.0); v.assign(n, 0.0); p.assign(n, 0.0);
    }
    void set(int i, int j, double r, double uu, double vv, double pp) {
        const size_t k = size_t(j) * nx + i;
        rho[k] = r; u[k] = uu; v[k] = vv; p[k] = pp;
    }
};

// The named test problems of main2d.cpp:52-135, same constants.
Problem setup(const std::string& test, int n) {
    Problem pr;
    if (test == "sod_x" || test == "sod_y") {
        const int m = 4;
        const bool along_x = (test == "sod_x");
        if (along_x) { pr.nx = n; pr.ny = m; pr.y_max = double(m) / n; }
        else { pr.nx = m; pr.ny = n; pr.x_max = double(m) / n; }
        pr.t_end = 0.2;
        pr.alloc();
        for (int j = 0; j < pr.ny; ++j)
            for (int i = 0; i < pr.nx; ++i) {
                const double s = along_x ? pr.xc(i) : pr.yc(j);
                if (s < 0.5) pr.set(i, j, 1.0, 0.0, 0.0, 1.0);
                else pr.set(i, j, 0.125, 0.0, 0.0, 0.1);
            }
    } else if (test == "lax_liu3") {  // Lax & Liu configuration 3
        pr.nx = pr.ny = n;
        pr.t_end = 0.3;
        pr.alloc();
        const double q[4][4] = {{1.5, 0.0, 0.0, 1.5},         // top right
                                {0.5323, 1.206, 0.0, 0.3},     // top left
                                {0.138, 1.206, 1.206, 0.029},  // bottom left
                                {0.5323, 0.0, 1.206, 0.3}};    // bottom right
        for (int j = 0; j < pr.ny; ++j)
            for (int i = 0; i < pr.nx; ++i) {
                const bool right = pr.xc(i) > 0.5, top = pr.yc(j) > 0.5;
                const double* W = top ? (right ? q[0] : q[1]) : (right ? q[3] : q[2]);
                pr.set(i, j, W[0], W[1], W[2], W[3]);
            }
    } else if (test == "sine2d") {  // smooth wave advected diagonally across the periodic box
        pr.nx = pr.ny = n;
        pr.bc_x = pr.bc_y = FV_BC_PERIODIC;
        pr.t_end = 1.0;
        pr.alloc();
        const double PI = 3.14159265358979323846;
        for (int j = 0; j < pr.ny; ++j)
            for (int i = 0; i < pr.nx; ++i)
                pr.set(i, j, 1.0 + 0.2 * std::sin(2.0 * PI * (pr.xc(i) + pr.yc(j))), 1.0, 1.0, 1.0);
    } else if (test == "kh") {  // smooth Kelvin-Helmholtz (McNally, Lyra & Passy 2012)
        pr.nx = pr.ny = n;
        pr.bc_x = pr.bc_y = FV_BC_PERIODIC;
        pr.t_end = 2.0;
        pr.alloc();
        const double PI = 3.14159265358979323846;
        const double rho1 = 1.0, rho2 = 2.0, rhom = 0.5 * (rho1 - rho2);
        const double u1 = 0.5, u2 = -0.5, um = 0.5 * (u1 - u2);
        const double L = 0.025;
        for (int j = 0; j < pr.ny; ++j)
            for (int i = 0; i < pr.nx; ++i) {
                const double x = pr.xc(i), y = pr.yc(j);
                double r, uu;
                if (y < 0.25) {
                    r = rho1 - rhom * std::exp((y - 0.25) / L);
                    uu = u1 - um * std::exp((y - 0.25) / L);
                } else if (y < 0.5) {
                    r = rho2 + rhom * std::exp((0.25 - y) / L);
                    uu = u2 + um * std::exp((0.25 - y) / L);
                } else if (y < 0.75) {
                    r = rho2 + rhom * std::exp((y - 0.75) / L);
                    uu = u2 + um * std::exp((y - 0.75) / L);
                } else {
                    r = rho1 - rhom * std::exp((0.75 - y) / L);
                    uu = u1 - um * std::exp((0.75 - y) / L);
                }
                pr.set(i, j, r, uu, 0.01 * std::sin(4.0 * PI * x), 2.5);
            }
    } else {
        std::cerr << "Unknown test '" << test << "' (use sod_x, sod_y, lax_liu3, sine2d or kh)\n";
        std::exit(1);
    }
    return pr;
}

int parse_bc(const std::string& s) {  // io_hdf5.hpp:157-161
    if (s == "periodic") return FV_BC_PERIODIC;
    if (s == "transmissive") return FV_BC_TRANSMISSIVE;
    throw std::runtime_error("unknown boundary condition '" + s + "'");
}
const char* bc_name(int bc) { return bc == FV_BC_PERIODIC ? "periodic" : "transmissive"; }

struct InitInfo {
    std::string test = "init";
    double t_end = -1.0;  // negative if the file does not give one
};

// read_initial_condition (io_hdf5.hpp:170-206): datasets rho, u, v, p of shape (ny, nx) and
// attributes nx, ny, x_min, x_max, y_min, y_max, bc_x, bc_y, optional t_end and test.  A snapshot
// file is therefore a valid initial condition (restart).
InitInfo read_initial_condition(const std::string& path, Problem& pr) {
    auto f = npz::read(path);
    auto need = [&](const char* k) -> const npz::Array& {
        auto it = f.find(k);
        if (it == f.end()) throw std::runtime_error(std::string("missing attribute ") + k);
        return it->second;
    };
    pr.nx = int(need("nx").scalar());
    pr.ny = int(need("ny").scalar());
    pr.x_min = need("x_min").scalar(); pr.x_max = need("x_max").scalar();
    pr.y_min = need("y_min").scalar(); pr.y_max = need("y_max").scalar();
    pr.bc_x = parse_bc(need("bc_x").str());
    pr.bc_y = parse_bc(need("bc_y").str());
    const size_t n = size_t(pr.nx) * pr.ny;
    auto field = [&](const char* k) {
        auto it = f.find(k);
        if (it == f.end()) throw std::runtime_error(std::string("missing dataset ") + k);
        if (it->second.count() != n) throw std::runtime_error(std::string("dataset ") + k + " has the wrong size");
        return it->second.doubles();
    };
    pr.rho = field("rho"); pr.u = field("u"); pr.v = field("v"); pr.p = field("p");
    InitInfo info;
    if (f.count("t_end")) info.t_end = f["t_end"].scalar();
    if (f.count("test")) info.test = f["test"].str();
    for (size_t k = 0; k < n; ++k)
        if (!(pr.rho[k] > 0.0) || !(pr.p[k] > 0.0))
            throw std::runtime_error("initial condition has non-positive density or pressure");
    return info;
}

struct RunInfo {  // io_hdf5.hpp:11-17
    std::string test, scheme, limiter;
    double cfl = 0.0;
    int step = 0;
};

// write_snapshot (io_hdf5.hpp:56-97): primitives of the interior cells in FP64, cell centres, and the
// run's attributes.  to_primitive is state2d.hpp:21-25, evaluated in the same order.
void write_snapshot(const std::string& path, const Problem& pr, const std::vector<double>& U, double t,
                    const RunInfo& info) {
    const size_t n = size_t(pr.nx) * pr.ny;
    std::vector<double> rho(n), u(n), v(n), p(n), x(pr.nx), y(pr.ny);
    for (size_t k = 0; k < n; ++k) {
        const double* c = &U[4 * k];
        const double uu = c[1] / c[0], vv = c[2] / c[0];
        rho[k] = c[0]; u[k] = uu; v[k] = vv;
        p[k] = (GAMMA - 1.0) * (c[3] - 0.5 * c[0] * (uu * uu + vv * vv));
    }
    for (int i = 0; i < pr.nx; ++i) x[i] = pr.xc(i);
    for (int j = 0; j < pr.ny; ++j) y[j] = pr.yc(j);
    const std::vector<size_t> d2{size_t(pr.ny), size_t(pr.nx)};
    npz::write(path, {{"rho", npz::f64(d2, rho.data())}, {"u", npz::f64(d2, u.data())}, {"v", npz::f64(d2, v.data())},
                      {"p", npz::f64(d2, p.data())}, {"x", npz::f64({size_t(pr.nx)}, x.data())},
                      {"y", npz::f64({size_t(pr.ny)}, y.data())}, {"t", npz::scalar(t)},
                      {"step", npz::scalar_int(info.step)}, {"gamma", npz::scalar(GAMMA)},
                      {"cfl", npz::scalar(info.cfl)}, {"nx", npz::scalar_int(pr.nx)}, {"ny", npz::scalar_int(pr.ny)},
                      {"x_min", npz::scalar(pr.x_min)}, {"x_max", npz::scalar(pr.x_max)},
                      {"y_min", npz::scalar(pr.y_min)}, {"y_max", npz::scalar(pr.y_max)},
                      {"bc_x", npz::string(bc_name(pr.bc_x))}, {"bc_y", npz::string(bc_name(pr.bc_y))},
                      {"test", npz::string(info.test)}, {"scheme", npz::string(info.scheme)},
                      {"limiter", npz::string(info.limiter)}});
}

// TrajectoryWriter::write (trajectory.hpp:53-91): t, one float32 U_<n> of shape (frames, 4, ny_c,
// nx_c) per storage size, and the run's attributes.
void write_trajectory(const std::string& path, const Problem& pr, const std::vector<int>& sizes,
                      const std::vector<std::vector<float>>& levels, const std::vector<double>& times,
                      const RunInfo& info, double t_end, double t_start) {
    std::vector<std::pair<std::string, npz::Array>> m;
    m.push_back({"t", npz::f64({times.size()}, times.data())});
    for (size_t l = 0; l < sizes.size(); ++l) {
        const int f = pr.nx / sizes[l];
        m.push_back({"U_" + std::to_string(sizes[l]),
                     npz::f32({times.size(), 4, size_t(pr.ny / f), size_t(sizes[l])}, levels[l].data())});
    }
    m.push_back({"variables", npz::string("rho, rho*u, rho*v, E")});
    m.push_back({"t_start", npz::scalar(t_start)});
    m.push_back({"t_end", npz::scalar(t_end)});
    m.push_back({"frames", npz::scalar_int(int(times.size()))});
    m.push_back({"steps", npz::scalar_int(info.step)});
    m.push_back({"gamma", npz::scalar(GAMMA)});
    m.push_back({"cfl", npz::scalar(info.cfl)});
    m.push_back({"solver_nx", npz::scalar_int(pr.nx)});
    m.push_back({"solver_ny", npz::scalar_int(pr.ny)});
    m.push_back({"x_min", npz::scalar(pr.x_min)}); m.push_back({"x_max", npz::scalar(pr.x_max)});
    m.push_back({"y_min", npz::scalar(pr.y_min)}); m.push_back({"y_max", npz::scalar(pr.y_max)});
    m.push_back({"bc_x", npz::string(bc_name(pr.bc_x))});
    m.push_back({"bc_y", npz::string(bc_name(pr.bc_y))});
    m.push_back({"test", npz::string(info.test)});
    m.push_back({"scheme", npz::string(info.scheme)});
    m.push_back({"limiter", npz::string(info.limiter)});
    npz::write(path, m);
}

// A failed library call: the reference exits 1 from report_bad_cell (solver2d.hpp:116-126) with the
// same message for a non-physical state.
[[noreturn]] void fail(int rc, const fv_bad_cell& bad) {
    if (rc == FV_ERR_NONPHYSICAL)
        std::cerr << "Non-physical state in cell (" << bad.i << ", " << bad.j << "): rho = " << bad.rho
                  << ", p = " << bad.p << '\n';
    else
        std::cerr << "euler2d: " << fv_last_error() << '\n';
    std::exit(1);
}

}  // namespace

int main(int argc, char* argv[]) {
    auto a = parse_args(argc, argv);
    const std::string test = a["test"], scheme = a["scheme"], lim_name = a["limiter"];
    const int n = std::atoi(a["n"].c_str()), nout = std::atoi(a["nout"].c_str());
    const double cfl = std::atof(a["cfl"].c_str());
    if (n <= 0 || nout <= 0 || !(cfl > 0.0)) { std::cerr << "n, nout and cfl must be positive\n"; return 1; }

    int flux;
    if (scheme == "rusanov") flux = FV_FLUX_RUSANOV;
    else if (scheme == "hllc") flux = FV_FLUX_HLLC;
    else { std::cerr << "Unknown scheme '" << scheme << "' (use rusanov or hllc)\n"; return 1; }

    int lim;
    if (lim_name == "none") lim = FV_LIM_NONE;
    else if (lim_name == "minmod") lim = FV_LIM_MINMOD;
    else if (lim_name == "vanleer") lim = FV_LIM_VANLEER;
    else if (lim_name == "unlimited") lim = FV_LIM_UNLIMITED;
    else { std::cerr << "Unknown limiter '" << lim_name << "'\n"; return 1; }

    Problem pr;
    std::string run_name = test;
    if (!a["init"].empty()) {
        InitInfo ii;
        try {
            ii = read_initial_condition(a["init"], pr);
        } catch (const std::exception& e) {
            std::cerr << "Error reading " << a["init"] << ": " << e.what() << '\n';
            return 1;
        }
        pr.t_end = ii.t_end;
        run_name = ii.test;
        if (pr.t_end <= 0.0 && a["tend"] == "default") {
            std::cerr << "The initial-condition file has no t_end; give one with --tend\n";
            return 1;
        }
    } else {
        pr = setup(test, n);
    }
    if (a["tend"] != "default") pr.t_end = std::atof(a["tend"].c_str());
    if (!(pr.t_end > 0.0)) { std::cerr << "tend must be positive\n"; return 1; }

    fv_solver* s = nullptr;
    fv_bad_cell bad{};
    int rc = fv_create(pr.nx, pr.ny, pr.x_min, pr.x_max, pr.y_min, pr.y_max, pr.bc_x, pr.bc_y, flux, lim, cfl,
                       nullptr, &s);
    if (rc != FV_OK) fail(rc, bad);
    if ((rc = fv_set_primitive(s, pr.rho.data(), pr.u.data(), pr.v.data(), pr.p.data())) != FV_OK) fail(rc, bad);
    if (a["profile"] == "yes") fv_profile(s, 1);

    RunInfo info{run_name, scheme, lim_name, cfl, 0};
    std::printf("%s: %d x %d cells, t_end = %g, %s + %s, CFL %g, 1 GPU\n", run_name.c_str(), pr.nx, pr.ny, pr.t_end,
                scheme.c_str(), lim_name.c_str(), cfl);

    const bool traj_mode = !a["traj"].empty();
    std::vector<int> sizes;
    std::string dir;
    if (traj_mode) {
        try {
            sizes = a["save"].empty() ? std::vector<int>{pr.nx} : parse_sizes(a["save"]);
            for (int m : sizes) {  // trajectory.hpp:19-28
                if (m <= 0 || pr.nx % m != 0)
                    throw std::runtime_error("save size " + std::to_string(m) + " does not divide nx = " +
                                             std::to_string(pr.nx));
                if (pr.ny % (pr.nx / m) != 0)
                    throw std::runtime_error("save size " + std::to_string(m) + " does not divide ny evenly");
            }
        } catch (const std::exception& e) {
            std::cerr << "Bad --save: " << e.what() << '\n';
            return 1;
        }
    } else {
        dir = a["out"] + "/" + run_name + "_" + scheme + "_" + lim_name + "_N" + std::to_string(pr.nx);
        std::filesystem::create_directories(dir);
    }

    const double t_start = std::atof(a["tstart"].c_str());
    if (!(t_start >= 0.0 && t_start < pr.t_end)) { std::cerr << "need 0 <= tstart < t_end\n"; return 1; }

    double t = 0.0;
    long long steps = 0;
    auto t0 = std::chrono::steady_clock::now();
    if (traj_mode) {
        // the whole --traj run (spin-up, frame 0, nout frames) in one call
        std::vector<std::vector<float>> levels(sizes.size());
        std::vector<float*> outs(sizes.size());
        for (size_t l = 0; l < sizes.size(); ++l) {
            const int f = pr.nx / sizes[l];
            levels[l].resize(size_t(nout + 1) * 4 * (pr.ny / f) * sizes[l]);
            outs[l] = levels[l].data();
        }
        std::vector<double> times(nout + 1);
        rc = fv_run_trajectory(s, t_start, pr.t_end, nout, sizes.data(), int(sizes.size()), outs.data(), times.data(),
                               &steps, &bad);
        if (rc != FV_OK) fail(rc, bad);
        t = times[nout];
        info.step = int(steps);
        try {
            write_trajectory(a["traj"], pr, sizes, levels, times, info, pr.t_end, t_start);
        } catch (const std::exception& e) {
            std::cerr << "Error writing trajectory: " << e.what() << '\n';
            return 1;
        }
    } else {
        std::vector<double> U(size_t(pr.nx) * pr.ny * 4);
        auto snapshot = [&](int k) {
            char buf[32];
            std::snprintf(buf, sizeof buf, "/snap_%04d.npz", k);
            if ((rc = fv_get_state(s, U.data())) != FV_OK) fail(rc, bad);
            try {
                write_snapshot(dir + buf, pr, U, t, info);
            } catch (const std::exception& e) {
                std::cerr << "Error writing snapshot: " << e.what() << '\n';
                std::exit(1);
            }
        };
        if (t_start > 0.0 && (rc = fv_advance_to(s, t_start, &t, &steps, &bad)) != FV_OK) fail(rc, bad);
        snapshot(0);
        for (int k = 1; k <= nout; ++k) {
            const double t_next = t_start + (pr.t_end - t_start) * k / nout;
            if ((rc = fv_advance_to(s, t_next, &t, &steps, &bad)) != FV_OK) fail(rc, bad);
            info.step = int(steps);
            snapshot(k);
            std::printf("  snapshot %2d/%d  t = %.4f  step %lld\n", k, nout, t, steps);
        }
    }

    const double secs = std::chrono::duration<double>(std::chrono::steady_clock::now() - t0).count();
    const double mcells = double(pr.nx) * pr.ny * double(steps) / secs / 1e6;
    std::printf("Done: %lld steps in %.2f s (%.2f million cell-updates per second). Output in %s\n", steps, secs,
                mcells, traj_mode ? a["traj"].c_str() : (dir + "/").c_str());
    if (a["profile"] == "yes") {
        double ms1 = 0, ms2 = 0;
        long long timed = 0;
        fv_profile_read(s, &ms1, &ms2, &timed);
        const double cells = double(pr.nx) * pr.ny;
        std::printf("\n%-30s %12s %12s\n", "stage kernel", "ms/launch", "ns per cell");
        std::printf("%-30s %12.4f %12.4f\n", "stage 1 (U1 = U + dt L(U))", ms1, 1e6 * ms1 / cells);
        std::printf("%-30s %12.4f %12.4f\n", "stage 2 (+ wave speeds)", ms2, 1e6 * ms2 / cells);
        std::printf("%-30s %12lld\n", "steps timed", timed);
    }
    fv_destroy(s);
    return 0;
}
