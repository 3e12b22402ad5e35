/*
 * CPU oracle for the 2D compressible-Euler finite-volume step (TEST INFRASTRUCTURE ONLY).
 *
 * This file is the checker, never the product: only tests/, __graft_entry__.smoke() and bench.py's
 * cpu_baseline / reference legs load it.  The product path (libfv, CUDA) never calls into it.
 *
 * It is a plain-C restatement of the reference solver core of GusGus2004/neural-pde-surrogate,
 * written from its published behaviour, with every operation in the same order and association
 * as the reference so that results are bit-identical when built without FMA contraction
 * (-ffp-contract=off).  Parity of this restatement is pinned two ways (tests/test_oracle_pin.py):
 * bit-for-bit against the reference's own headers compiled in oracle/_ref (when present), and
 * against golden fixtures in tests/golden/ generated from that build.
 *
 * Layout: the caller passes interior cells only, row-major, 4 doubles per cell (rho, rho*u, rho*v, E),
 * i.e. U[(j*nx + i)*4 + q].  Internally the ghosted layout of the reference is used
 * (solver/src/grid2d.hpp:12-28): (ny+4) x (nx+4) cells with a 2-cell ghost ring.
 */
#include <math.h>
#include <stdint.h>
#include <stdlib.h>
#include <string.h>
#ifdef _OPENMP
#include <omp.h>
#endif

#define ORC_GAMMA 1.4 /* solver/src/state2d.hpp:7 */
#define NG 2

enum { ORC_BC_TRANSMISSIVE = 0, ORC_BC_PERIODIC = 1 };
enum { ORC_FLUX_RUSANOV = 0, ORC_FLUX_HLLC = 1 };
enum { ORC_LIM_NONE = 0, ORC_LIM_UNLIMITED = 1, ORC_LIM_MINMOD = 2, ORC_LIM_VANLEER = 3 };

typedef struct { double rho, mx, my, E; } cons_t;  /* state2d.hpp:9 */
typedef struct { double rho, u, v, p; } prim_t;    /* state2d.hpp:10 */

/* std::min / std::max semantics (the reference uses <algorithm>): min(a,b) = (b<a)?b:a, max = (a<b)?b:a */
static inline double smin(double a, double b) { return (b < a) ? b : a; }
static inline double smax(double a, double b) { return (a < b) ? b : a; }

/* state2d.hpp:16-19 */
static inline cons_t to_conserved(prim_t W) {
    cons_t U;
    U.rho = W.rho;
    U.mx = W.rho * W.u;
    U.my = W.rho * W.v;
    U.E = W.p / (ORC_GAMMA - 1.0) + 0.5 * W.rho * (W.u * W.u + W.v * W.v);
    return U;
}

/* state2d.hpp:21-25 */
static inline prim_t to_primitive(cons_t U) {
    prim_t W;
    double u = U.mx / U.rho, v = U.my / U.rho;
    double p = (ORC_GAMMA - 1.0) * (U.E - 0.5 * U.rho * (u * u + v * v));
    W.rho = U.rho; W.u = u; W.v = v; W.p = p;
    return W;
}

/* state2d.hpp:27 */
static inline double sound_speed(prim_t W) { return sqrt(ORC_GAMMA * W.p / W.rho); }

/* state2d.hpp:30-36 */
static inline cons_t flux_x(cons_t U) {
    prim_t W = to_primitive(U);
    cons_t F;
    F.rho = U.mx;
    F.mx = U.mx * W.u + W.p;
    F.my = U.my * W.u;
    F.E = W.u * (U.E + W.p);
    return F;
}

/* state2d.hpp:39 */
static inline cons_t swap_xy(cons_t U) { cons_t S = {U.rho, U.my, U.mx, U.E}; return S; }

/* state2d.hpp:12-14 (componentwise operators) */
static inline cons_t c_add(cons_t a, cons_t b) { cons_t r = {a.rho + b.rho, a.mx + b.mx, a.my + b.my, a.E + b.E}; return r; }
static inline cons_t c_sub(cons_t a, cons_t b) { cons_t r = {a.rho - b.rho, a.mx - b.mx, a.my - b.my, a.E - b.E}; return r; }
static inline cons_t c_scale(double s, cons_t a) { cons_t r = {s * a.rho, s * a.mx, s * a.my, s * a.E}; return r; }

/* riemann2d.hpp:11-15 */
static cons_t rusanov_flux(cons_t UL, cons_t UR) {
    prim_t WL = to_primitive(UL), WR = to_primitive(UR);
    double s_max = smax(fabs(WL.u) + sound_speed(WL), fabs(WR.u) + sound_speed(WR));
    return c_sub(c_scale(0.5, c_add(flux_x(UL), flux_x(UR))), c_scale(0.5 * s_max, c_sub(UR, UL)));
}

/* riemann2d.hpp:18-24 (Toro eq. 10.39) */
static cons_t hllc_star_state(cons_t U, prim_t W, double S, double S_star) {
    double factor = W.rho * (S - W.u) / (S - S_star);
    cons_t r;
    r.rho = factor;
    r.mx = factor * S_star;
    r.my = factor * W.v;
    r.E = factor * (U.E / W.rho + (S_star - W.u) * (S_star + W.p / (W.rho * (S - W.u))));
    return r;
}

/* riemann2d.hpp:27-39, Davis wave speeds */
static cons_t hllc_flux(cons_t UL, cons_t UR) {
    prim_t WL = to_primitive(UL), WR = to_primitive(UR);
    double aL = sound_speed(WL), aR = sound_speed(WR);
    double SL = smin(WL.u - aL, WR.u - aR);
    double SR = smax(WL.u + aL, WR.u + aR);
    double S_star = (WR.p - WL.p + WL.rho * WL.u * (SL - WL.u) - WR.rho * WR.u * (SR - WR.u))
                  / (WL.rho * (SL - WL.u) - WR.rho * (SR - WR.u));
    if (0.0 <= SL) return flux_x(UL);
    if (0.0 <= S_star) return c_add(flux_x(UL), c_scale(SL, c_sub(hllc_star_state(UL, WL, SL, S_star), UL)));
    if (0.0 <= SR) return c_add(flux_x(UR), c_scale(SR, c_sub(hllc_star_state(UR, WR, SR, S_star), UR)));
    return flux_x(UR);
}

static inline cons_t flux_fn(int flux, cons_t UL, cons_t UR) {
    return flux == ORC_FLUX_HLLC ? hllc_flux(UL, UR) : rusanov_flux(UL, UR);
}

/* riemann2d.hpp:42-44: rotate so y becomes x, solve, rotate back */
static inline cons_t flux_y_face(int flux, cons_t UL, cons_t UR) {
    return swap_xy(flux_fn(flux, swap_xy(UL), swap_xy(UR)));
}

/* limiters.hpp:7-18 */
static inline double limiter(int lim, double a, double b) {
    switch (lim) {
    case ORC_LIM_NONE: return 0.0;
    case ORC_LIM_UNLIMITED: return 0.5 * (a + b);
    case ORC_LIM_MINMOD:
        if (a * b <= 0.0) return 0.0;
        return (fabs(a) < fabs(b)) ? a : b;
    default: /* van Leer */
        if (a * b <= 0.0) return 0.0;
        return 2.0 * a * b / (a + b);
    }
}

/* solver2d.hpp:17-22 */
static inline prim_t limited_slope(prim_t Wm, prim_t W0, prim_t Wp, int lim) {
    prim_t s;
    s.rho = limiter(lim, W0.rho - Wm.rho, Wp.rho - W0.rho);
    s.u = limiter(lim, W0.u - Wm.u, Wp.u - W0.u);
    s.v = limiter(lim, W0.v - Wm.v, Wp.v - W0.v);
    s.p = limiter(lim, W0.p - Wm.p, Wp.p - W0.p);
    return s;
}

/* solver2d.hpp:25-27 */
static inline prim_t edge(prim_t W, prim_t dW, double s) {
    prim_t e;
    e.rho = W.rho + 0.5 * s * dW.rho;
    e.u = W.u + 0.5 * s * dW.u;
    e.v = W.v + 0.5 * s * dW.v;
    e.p = W.p + 0.5 * s * dW.p;
    return e;
}

/* ------------------------------------------------------------------------------------------------ */

typedef struct {
    int nx, ny;
    double x_min, x_max, y_min, y_max, dx, dy;
    int bc_x, bc_y, flux, lim;
    double cfl;
    cons_t *U, *U1, *L, *G; /* ghosted U, U1, L; G is nx*(ny+1) (solver2d.hpp:110-112) */
    prim_t *W, *dW;
} orc_solver;

static inline int gidx(const orc_solver* s, int i, int j) { return (j + NG) * (s->nx + 2 * NG) + (i + NG); }
static inline int gsize(const orc_solver* s) { return (s->nx + 2 * NG) * (s->ny + 2 * NG); }

/* grid2d.hpp:30-39 (make_grid) + solver2d.hpp:61-64 (allocation once in the constructor) */
orc_solver* orc_create(int nx, int ny, double x_min, double x_max, double y_min, double y_max,
                       int bc_x, int bc_y, int flux, int lim, double cfl) {
    if (nx <= 0 || ny <= 0) return NULL;
    orc_solver* s = (orc_solver*)calloc(1, sizeof(orc_solver));
    s->nx = nx; s->ny = ny;
    s->x_min = x_min; s->x_max = x_max; s->y_min = y_min; s->y_max = y_max;
    s->dx = (x_max - x_min) / nx;
    s->dy = (y_max - y_min) / ny;
    s->bc_x = bc_x; s->bc_y = bc_y; s->flux = flux; s->lim = lim; s->cfl = cfl;
    size_t n = (size_t)gsize(s);
    s->U = (cons_t*)calloc(n, sizeof(cons_t));
    s->U1 = (cons_t*)calloc(n, sizeof(cons_t));
    s->L = (cons_t*)calloc(n, sizeof(cons_t));
    s->W = (prim_t*)calloc(n, sizeof(prim_t));
    s->dW = (prim_t*)calloc(n, sizeof(prim_t));
    s->G = (cons_t*)calloc((size_t)nx * (ny + 1), sizeof(cons_t));
    return s;
}

void orc_destroy(orc_solver* s) {
    if (!s) return;
    free(s->U); free(s->U1); free(s->L); free(s->W); free(s->dW); free(s->G); free(s);
}

double orc_dx(const orc_solver* s) { return s->dx; }
double orc_dy(const orc_solver* s) { return s->dy; }

void orc_set_state(orc_solver* s, const double* U) {
    for (int j = 0; j < s->ny; ++j)
        for (int i = 0; i < s->nx; ++i) memcpy(&s->U[gidx(s, i, j)], U + ((size_t)j * s->nx + i) * 4, 32);
}

void orc_get_state(const orc_solver* s, double* U) {
    for (int j = 0; j < s->ny; ++j)
        for (int i = 0; i < s->nx; ++i) memcpy(U + ((size_t)j * s->nx + i) * 4, &s->U[gidx(s, i, j)], 32);
}

/* Primitive (rho, u, v, p), each (ny, nx) -> conserved interior (io_hdf5.hpp:197-204 / to_conserved). */
void orc_primitive_to_state(int n, const double* rho, const double* u, const double* v, const double* p, double* U) {
    for (int k = 0; k < n; ++k) {
        prim_t W = {rho[k], u[k], v[k], p[k]};
        cons_t c = to_conserved(W);
        memcpy(U + (size_t)k * 4, &c, 32);
    }
}

/* grid2d.hpp:43-66: x-ghosts on physical rows, then y-ghosts over whole rows (corners included) */
static void apply_bcs(const orc_solver* s, cons_t* U) {
    const int nx = s->nx, ny = s->ny;
    for (int j = 0; j < ny; ++j)
        for (int k = 1; k <= NG; ++k) {
            if (s->bc_x == ORC_BC_PERIODIC) {
                U[gidx(s, -k, j)] = U[gidx(s, nx - k, j)];
                U[gidx(s, nx - 1 + k, j)] = U[gidx(s, k - 1, j)];
            } else {
                U[gidx(s, -k, j)] = U[gidx(s, 0, j)];
                U[gidx(s, nx - 1 + k, j)] = U[gidx(s, nx - 1, j)];
            }
        }
    for (int i = -NG; i < nx + NG; ++i)
        for (int k = 1; k <= NG; ++k) {
            if (s->bc_y == ORC_BC_PERIODIC) {
                U[gidx(s, i, -k)] = U[gidx(s, i, ny - k)];
                U[gidx(s, i, ny - 1 + k)] = U[gidx(s, i, k - 1)];
            } else {
                U[gidx(s, i, -k)] = U[gidx(s, i, 0)];
                U[gidx(s, i, ny - 1 + k)] = U[gidx(s, i, ny - 1)];
            }
        }
}

/* Ghost fill on a caller-provided ghosted array (test hook for the grid2d known answers). */
void orc_apply_bcs_ghosted(int nx, int ny, int bc_x, int bc_y, double* Ug) {
    orc_solver tmp;
    memset(&tmp, 0, sizeof tmp);
    tmp.nx = nx; tmp.ny = ny; tmp.bc_x = bc_x; tmp.bc_y = bc_y;
    apply_bcs(&tmp, (cons_t*)Ug);
}

/* solver2d.hpp:67-83 (+ report_bad_cell :116-126 without the exit: the first row-major bad cell is
 * returned instead).  Returns 0 and *dt on success, 1 on a non-physical state. */
int orc_compute_dt(const orc_solver* s, double* dt, int* bad_i, int* bad_j, double* bad_rho, double* bad_p) {
    double sx = 0.0, sy = 0.0;
    int bad = 0;
#pragma omp parallel for reduction(max : sx, sy) reduction(|| : bad)
    for (int j = 0; j < s->ny; ++j)
        for (int i = 0; i < s->nx; ++i) {
            prim_t Wc = to_primitive(s->U[gidx(s, i, j)]);
            if (!(Wc.rho > 0.0) || !(Wc.p > 0.0)) { bad = 1; continue; }
            double a = sound_speed(Wc);
            sx = smax(sx, fabs(Wc.u) + a);
            sy = smax(sy, fabs(Wc.v) + a);
        }
    if (bad) {
        for (int j = 0; j < s->ny; ++j)
            for (int i = 0; i < s->nx; ++i) {
                prim_t Wc = to_primitive(s->U[gidx(s, i, j)]);
                if (!(Wc.rho > 0.0) || !(Wc.p > 0.0)) {
                    if (bad_i) *bad_i = i;
                    if (bad_j) *bad_j = j;
                    if (bad_rho) *bad_rho = Wc.rho;
                    if (bad_p) *bad_p = Wc.p;
                    return 1;
                }
            }
    }
    *dt = s->cfl / (sx / s->dx + sy / s->dy);
    return 0;
}

/* solver2d.hpp:129-180 */
static void compute_rhs(orc_solver* s, cons_t* U) {
    const int nx = s->nx, ny = s->ny, n = gsize(s), lim = s->lim, flux = s->flux;
    cons_t* L = s->L;
    prim_t *W = s->W, *dW = s->dW;
    cons_t* G = s->G;
    apply_bcs(s, U);
#pragma omp parallel for
    for (int k = 0; k < n; ++k) W[k] = to_primitive(U[k]);

    /* x-direction: each row j only touches its own cells (solver2d.hpp:139-152) */
#pragma omp parallel for
    for (int j = 0; j < ny; ++j) {
        for (int i = 0; i < nx; ++i) { cons_t z = {0.0, 0.0, 0.0, 0.0}; L[gidx(s, i, j)] = z; }
        for (int i = -1; i <= nx; ++i)
            dW[gidx(s, i, j)] = limited_slope(W[gidx(s, i - 1, j)], W[gidx(s, i, j)], W[gidx(s, i + 1, j)], lim);
        for (int i = 0; i <= nx; ++i) {
            int kl = gidx(s, i - 1, j), kr = gidx(s, i, j);
            cons_t F = flux_fn(flux, to_conserved(edge(W[kl], dW[kl], +1.0)), to_conserved(edge(W[kr], dW[kr], -1.0)));
            if (i > 0) L[kl] = c_sub(L[kl], c_scale(1.0 / s->dx, F));
            if (i < nx) L[kr] = c_add(L[kr], c_scale(1.0 / s->dx, F));
        }
    }

    /* y-direction: slopes, face fluxes into G, then each row collects its two fluxes (:156-178) */
#pragma omp parallel for
    for (int j = -1; j <= ny; ++j)
        for (int i = 0; i < nx; ++i)
            dW[gidx(s, i, j)] = limited_slope(W[gidx(s, i, j - 1)], W[gidx(s, i, j)], W[gidx(s, i, j + 1)], lim);
#pragma omp parallel for
    for (int j = 0; j <= ny; ++j)
        for (int i = 0; i < nx; ++i) {
            int kb = gidx(s, i, j - 1), kt = gidx(s, i, j);
            G[(size_t)j * nx + i] = flux_y_face(flux, to_conserved(edge(W[kb], dW[kb], +1.0)),
                                                to_conserved(edge(W[kt], dW[kt], -1.0)));
        }
#pragma omp parallel for
    for (int j = 0; j < ny; ++j)
        for (int i = 0; i < nx; ++i) {
            int k = gidx(s, i, j);
            L[k] = c_add(L[k], c_scale(1.0 / s->dy, G[(size_t)j * nx + i]));
            L[k] = c_sub(L[k], c_scale(1.0 / s->dy, G[(size_t)(j + 1) * nx + i]));
        }
}

/* solver2d.hpp:86-103: SSP-RK2 (Heun) */
void orc_step(orc_solver* s, double dt) {
    const int nx = s->nx, ny = s->ny;
    cons_t *U = s->U, *U1 = s->U1, *L = s->L;
    compute_rhs(s, U);
#pragma omp parallel for
    for (int j = 0; j < ny; ++j)
        for (int i = 0; i < nx; ++i) {
            int k = gidx(s, i, j);
            U1[k] = c_add(U[k], c_scale(dt, L[k]));
        }
    compute_rhs(s, U1);
#pragma omp parallel for
    for (int j = 0; j < ny; ++j)
        for (int i = 0; i < nx; ++i) {
            int k = gidx(s, i, j);
            U[k] = c_scale(0.5, c_add(c_add(U[k], U1[k]), c_scale(dt, L[k])));
        }
}

/* Time loop of the driver (main2d.cpp:236-242): advance until t >= t_next, landing exactly on t_next.
 * Returns 0, or 1 on a non-physical state (state left as it was before the failing step). */
int orc_advance_to(orc_solver* s, double t_next, double* t, long long* steps,
                   int* bad_i, int* bad_j, double* bad_rho, double* bad_p) {
    while (*t < t_next) {
        double dt;
        if (orc_compute_dt(s, &dt, bad_i, bad_j, bad_rho, bad_p)) return 1;
        dt = smin(dt, t_next - *t);
        orc_step(s, dt);
        *t += dt;
        ++*steps;
    }
    return 0;
}

/* Frame time of the driver (main2d.cpp:236): t_start + (t_end - t_start) * k / nout */
double orc_frame_time(double t_start, double t_end, int k, int nout) {
    return t_start + (t_end - t_start) * k / nout;
}

/* TrajectoryWriter::add for one level (trajectory.hpp:31-51): f x f block sums in FP64, j-outer /
 * i-inner, times 1/(f*f), cast to float; layout (variable, y, x). */
void orc_block_average(const orc_solver* s, int f, float* out) {
    const int nxc = s->nx / f, nyc = s->ny / f;
    const double inv = 1.0 / ((double)f * f);
    for (int jc = 0; jc < nyc; ++jc)
        for (int ic = 0; ic < nxc; ++ic) {
            double acc[4] = {0.0, 0.0, 0.0, 0.0};
            for (int j = jc * f; j < (jc + 1) * f; ++j)
                for (int i = ic * f; i < (ic + 1) * f; ++i) {
                    const cons_t* c = &s->U[gidx(s, i, j)];
                    acc[0] += c->rho; acc[1] += c->mx; acc[2] += c->my; acc[3] += c->E;
                }
            for (int q = 0; q < 4; ++q) out[((size_t)q * nyc + jc) * nxc + ic] = (float)(acc[q] * inv);
        }
}

/* Single-face hooks for the Riemann known answers (test_riemann2d.cpp). */
void orc_flux(int flux, const double* UL, const double* UR, double* F) {
    cons_t a, b;
    memcpy(&a, UL, 32); memcpy(&b, UR, 32);
    cons_t r = flux_fn(flux, a, b);
    memcpy(F, &r, 32);
}
void orc_flux_y(int flux, const double* UL, const double* UR, double* F) {
    cons_t a, b;
    memcpy(&a, UL, 32); memcpy(&b, UR, 32);
    cons_t r = flux_y_face(flux, a, b);
    memcpy(F, &r, 32);
}
void orc_flux_x_physical(const double* U, double* F) {
    cons_t a;
    memcpy(&a, U, 32);
    cons_t r = flux_x(a);
    memcpy(F, &r, 32);
}
void orc_to_conserved(const double* W, double* U) {
    prim_t w;
    memcpy(&w, W, 32);
    cons_t r = to_conserved(w);
    memcpy(U, &r, 32);
}

/* 1D HLLC (solver/src/riemann.hpp:27-43, state.hpp): the reference's own 1D flux, used by its
 * test_riemann2d.cpp:21-31 as the comparison for the 2D flux at v = 0.  U = (rho, rho*u, E). */
void orc_hllc_1d(const double* UL, const double* UR, double* F) {
    double rl = UL[0], ul = UL[1] / UL[0], pl = (ORC_GAMMA - 1.0) * (UL[2] - 0.5 * UL[0] * ul * ul);
    double rr = UR[0], ur = UR[1] / UR[0], pr = (ORC_GAMMA - 1.0) * (UR[2] - 0.5 * UR[0] * ur * ur);
    double aL = sqrt(ORC_GAMMA * pl / rl), aR = sqrt(ORC_GAMMA * pr / rr);
    double SL = smin(ul - aL, ur - aR), SR = smax(ul + aL, ur + aR);
    double S_star = (pr - pl + rl * ul * (SL - ul) - rr * ur * (SR - ur)) / (rl * (SL - ul) - rr * (SR - ur));
    double FL[3] = {UL[1], UL[1] * ul + pl, ul * (UL[2] + pl)};
    double FR[3] = {UR[1], UR[1] * ur + pr, ur * (UR[2] + pr)};
    if (0.0 <= SL) { memcpy(F, FL, 24); return; }
    if (0.0 <= S_star || 0.0 <= SR) {
        int left = 0.0 <= S_star;
        const double* Uk = left ? UL : UR;
        const double* Fk = left ? FL : FR;
        double rk = left ? rl : rr, uk = left ? ul : ur, pk = left ? pl : pr, S = left ? SL : SR;
        double factor = rk * (S - uk) / (S - S_star);
        double st[3] = {factor, factor * S_star,
                        factor * (Uk[2] / rk + (S_star - uk) * (S_star + pk / (rk * (S - uk))))};
        for (int q = 0; q < 3; ++q) F[q] = Fk[q] + S * (st[q] - Uk[q]);
        return;
    }
    memcpy(F, FR, 24);
}

int orc_max_threads(void) {
#ifdef _OPENMP
    return omp_get_max_threads();
#else
    return 1;
#endif
}
