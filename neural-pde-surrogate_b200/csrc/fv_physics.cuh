// Device-side physics of the 2D Euler finite-volume step: equation of state, slope limiters, MUSCL
// edge states and the Rusanov / HLLC face fluxes.
//
// Every expression keeps the operation order and association of the reference solver core
// (GusGus2004/neural-pde-surrogate, solver/src/{state2d,limiters,riemann2d,solver2d}.hpp) so that,
// compiled with --fmad=false, results are bit-identical to the reference's CPU build (which uses no
// FMA contraction).  IEEE division and square root (CUDA's default `/` and `sqrt` for double) are
// used; replacing a division with a reciprocal multiply would change the bits.
#pragma once
#include <cstdint>

namespace fv {

constexpr double GAMMA = 1.4;          // state2d.hpp:7
constexpr double GM1 = GAMMA - 1.0;    // the double constant 0.39999999999999991 used by the reference

enum : int { BC_TRANSMISSIVE = 0, BC_PERIODIC = 1 };
enum : int { FLUX_RUSANOV = 0, FLUX_HLLC = 1 };
enum : int { LIM_NONE = 0, LIM_UNLIMITED = 1, LIM_MINMOD = 2, LIM_VANLEER = 3 };

// One cell: conserved (rho, rho*u, rho*v, E) or primitive (rho, u, v, p).  32 bytes, the same layout
// as the reference's e2d::Conserved / e2d::Primitive (state2d.hpp:9-10).
struct __align__(16) Q4 {
    double a, b, c, d;
};

__device__ __forceinline__ Q4 ld_q4(const Q4* p) {
    const double2* v = reinterpret_cast<const double2*>(p);
    double2 x = v[0], y = v[1];
    return Q4{x.x, x.y, y.x, y.y};
}
__device__ __forceinline__ void st_q4(Q4* p, const Q4& q) {
    double2* v = reinterpret_cast<double2*>(p);
    v[0] = make_double2(q.a, q.b);
    v[1] = make_double2(q.c, q.d);
}
__device__ __forceinline__ Q4 ldg_q4(const Q4* p) {
    const double2* v = reinterpret_cast<const double2*>(p);
    double2 x = __ldg(v), y = __ldg(v + 1);
    return Q4{x.x, x.y, y.x, y.y};
}

// std::min / std::max as the reference uses them (<algorithm>): min(a,b) = (b<a)?b:a, max(a,b) = (a<b)?b:a.
__device__ __forceinline__ double smin(double a, double b) { return (b < a) ? b : a; }
__device__ __forceinline__ double smax(double a, double b) { return (a < b) ? b : a; }

// Magnitude tests from the exponent field (integer compares, which leave the FP64 pipe free):
// mag_in<LO, HI>(x): 2^LO <= |x| < 2^HI; pos_in<LO, HI>(x): 2^LO <= x < 2^HI (x positive).  Zeros,
// subnormals, infinities and NaN fail both.  The high word of |x| orders like |x| on exponent
// boundaries, and a negative x has the sign bit set, which puts it above the range as unsigned.
template <int LO, int HI>
__device__ __forceinline__ bool mag_in(double x) {
    static_assert(LO < HI && 1023 + LO > 0 && 1023 + HI < 2047, "exponent range");
    const unsigned h = unsigned(__double2hiint(x)) & 0x7fffffffu;
    return h - unsigned((1023 + LO) << 20) < unsigned((HI - LO) << 20);
}
template <int LO, int HI>
__device__ __forceinline__ bool pos_in(double x) {
    static_assert(LO < HI && 1023 + LO > 0 && 1023 + HI < 2047, "exponent range");
    return unsigned(__double2hiint(x)) - unsigned((1023 + LO) << 20) < unsigned((HI - LO) << 20);
}

// ---- two correctly rounded divisions for special operands ------------------------------------
// Both return exactly the IEEE round-to-nearest quotient (what `/` returns) for every finite input;
// outside the ranges where their reasoning holds they fall back to `/`.

// p / (GAMMA - 1.0) with one multiply and two FMAs: Markstein's correction step (P. Markstein,
// "Computation of elementary functions on the IBM RISC System/6000 processor", IBM J. Res. Dev.
// 34(1), 1990): with y = RN(1/b) and q0 within one ulp of a/b, r = a - q0*b is exact and
// RN(q0 + r*y) = RN(a/b).  For b = GAMMA-1, y*b differs from 1 by 0.4 * 2^-53, so q0 = RN(a*y) is
// within 0.9 ulp of a/b and the theorem applies.
constexpr double Y_GM1 = 1.0 / GM1;  // RN(1/(GAMMA-1)) = 2.5000000000000004
__device__ __forceinline__ double div_gm1(double p) {
    if (!mag_in<-899, 900>(p)) return p / GM1;  // zero, subnormal, huge, inf, NaN
    const double q0 = p * Y_GM1;
    const double r = fma(-q0, GM1, p);
    return fma(r, Y_GM1, q0);
}

// a / b at every general division site below: the IEEE quotient in the parity build.
#ifndef FV_TOLERANCE_BUILD
__device__ __forceinline__ double fdiv(double a, double b) { return a / b; }
#else
// The tolerance build (FMA contraction; 1e-12 relative per step and 1e-9 per run of the parity build
// allowed): a seed y ~ 1/b from the approximate reciprocal instruction, one Newton-Raphson step
// y + y(1 - b y), q0 = a y, and Markstein's correction q0 + (a - q0 b) y (the method cited above).
// Emulated on a CPU with seeds of relative error up to 2^-20 this gave the correctly rounded
// quotient for all of 2e7 random operand pairs, and at most 1 ulp from 2^-14 seeds.  Operands
// outside 2^-499 <= |a|, |b| < 2^500 take `/`: zeros (so that a signed zero keeps IEEE's sign),
// infinities, NaN, and the extremes whose quotient could be subnormal or overflow.
__device__ __forceinline__ double fdiv(double a, double b) {
    if (!(mag_in<-499, 500>(a) && mag_in<-499, 500>(b))) return a / b;
    double y;
    asm("rcp.approx.ftz.f64 %0, %1;" : "=d"(y) : "d"(b));
    y = fma(y, fma(-b, y, 1.0), y);
    const double q = a * y;
    return fma(fma(-q, b, a), y, q);
}
// 1/b for divisions that share a denominator: the same seed and two Newton-Raphson steps (a quotient
// a * recip(b) is then within about 1.5 ulp); operands outside 2^-499 <= |b| < 2^500 take `/`.
__device__ __forceinline__ double recip(double b) {
    if (!mag_in<-499, 500>(b)) return 1.0 / b;
    double y;
    asm("rcp.approx.ftz.f64 %0, %1;" : "=d"(y) : "d"(b));
    y = fma(y, fma(-b, y, 1.0), y);
    return fma(y, fma(-b, y, 1.0), y);
}
#endif

// a / b with a fast path for a zero numerator (zero velocities in a fluid at rest, equal left and
// right states at a face): IEEE gives +-0 / b = +-0 with the sign of a XOR the sign of b for every
// nonzero, non-NaN b (infinities included), which is a * copysign(1, b) exactly.  The general
// division routine treats a zero numerator as a special case and runs ~3x slower on it.
__device__ __forceinline__ double div_z(double a, double b) {
    if ((__double_as_longlong(a) << 1) == 0 && b != 0.0 && b == b) return a * copysign(1.0, b);  // a = +-0
    return fdiv(a, b);
}

// RN(m / rho) for m = RN(rho * u): the velocity to_primitive recovers from a momentum that
// to_conserved formed from the same rho and u.  Every face state of the reference takes that round
// trip (to_conserved(edge(...)) then to_primitive, solver2d.hpp:145-148,165-169 with
// riemann2d.hpp:12,28), so the quotient can be decided without dividing.  e = rho*u - m is exact
// (one fma: the error-free product of Dekker, and of Ogita, Rump and Oishi, SIAM J. Sci. Comput.
// 26(6), 2005), so the exact quotient is m/rho = u - e/rho, and |e/rho| <= 2^-53 |u| (1 + 2^-53) <
// ulp(u).  Its correctly rounded value is u when |e/rho| < ulp(u)/2, else the neighbour of u on the
// side of -e/rho.  No tie can occur: the exact quotient of two doubles is never halfway between two
// doubles.  When u is a power of two the product is exact and e = 0.  The bound 2^-299 <= rho, |u| <
// 2^300 keeps e, rho*ulp(u)/2 and rho*u normal; outside it (a zero, negative or extreme density, a
// zero or extreme velocity) the division is done.  e is nonzero past the first test, so its sign
// and u's compare as sign bits.
__device__ __forceinline__ double div_back(double m, double rho, double u) {
    if (!(pos_in<-299, 300>(rho) && mag_in<-299, 300>(u))) return div_z(m, rho);
    const double e = fma(rho, u, -m);
    const double half_ulp = __hiloint2double((__double2hiint(u) & 0x7ff00000) - (53 << 20), 0);  // 2^(k-53)
    if (fabs(e) < rho * half_ulp) return u;
    const long long bits = __double_as_longlong(u);
    const bool same_sign = (__double2hiint(e) ^ __double2hiint(u)) >= 0;
    return __longlong_as_double(same_sign ? bits - 1 : bits + 1);  // toward zero if same sign
}

// state2d.hpp:16-19 (p / (GAMMA - 1.0) through div_gm1: same bits, fewer instructions)
__device__ __forceinline__ Q4 to_conserved(const Q4& W) {
    return Q4{W.a, W.a * W.b, W.a * W.c, div_gm1(W.d) + 0.5 * W.a * (W.b * W.b + W.c * W.c)};
}

// state2d.hpp:21-25
__device__ __forceinline__ Q4 to_primitive(const Q4& U) {
#ifndef FV_TOLERANCE_BUILD
    double u = div_z(U.b, U.a), v = div_z(U.c, U.a);
#else
    const double r = recip(U.a);  // one reciprocal for both velocities
    double u = U.b * r, v = U.c * r;
#endif
    double p = GM1 * (U.d - 0.5 * U.a * (u * u + v * v));
    return Q4{U.a, u, v, p};
}

// state2d.hpp:27
__device__ __forceinline__ double sound_speed(const Q4& W) { return sqrt(fdiv(GAMMA * W.d, W.a)); }

// One side of a face: U = to_conserved(We) of the MUSCL edge state We, W = to_primitive(U), the
// primitive state the reference's flux function recomputes from U (riemann2d.hpp:12,28), and its
// sound speed a = sound_speed(W), which both flux functions evaluate once per side (riemann2d.hpp:13,
// 29).  The velocities come from div_back (same bits as the divisions of to_primitive); the pressure
// and the sound speed are the reference's expressions on them.  The tolerance build keeps the edge
// state itself as W (within an ulp per component of the round trip), and r = 1/rho is shared by
// the side's divisions by rho.
struct FaceSide {
    Q4 U, W;
    double a, r;  // r: tolerance build only
};
__device__ __forceinline__ FaceSide face_side(const Q4& We) {
    const Q4 U = to_conserved(We);
#ifndef FV_TOLERANCE_BUILD
    const double u = div_back(U.b, We.a, We.b), v = div_back(U.c, We.a, We.c);
    const Q4 W{U.a, u, v, GM1 * (U.d - 0.5 * U.a * (u * u + v * v))};
    return FaceSide{U, W, sound_speed(W), 0.0};
#else
    const double r = recip(We.a);
    return FaceSide{U, We, sqrt(GAMMA * We.d * r), r};
#endif
}

// state2d.hpp:30-36, with the primitive state of U supplied by the caller (it is the same
// to_primitive(U) the reference recomputes, so reusing it is bit-identical).
__device__ __forceinline__ Q4 flux_x(const Q4& U, const Q4& W) {
    return Q4{U.b, U.b * W.b + W.d, U.c * W.b, W.b * (U.d + W.d)};
}

// limiters.hpp:7-18
template <int LIM>
__device__ __forceinline__ double limiter(double a, double b) {
    if constexpr (LIM == LIM_NONE) {
        return 0.0;
    } else if constexpr (LIM == LIM_UNLIMITED) {
        return 0.5 * (a + b);
    } else if constexpr (LIM == LIM_MINMOD) {
        if (a * b <= 0.0) return 0.0;
        return (fabs(a) < fabs(b)) ? a : b;
    } else {
        if (a * b <= 0.0) return 0.0;
        return fdiv(2.0 * a * b, a + b);
    }
}

// solver2d.hpp:17-22
template <int LIM>
__device__ __forceinline__ Q4 limited_slope(const Q4& Wm, const Q4& W0, const Q4& Wp) {
    return Q4{limiter<LIM>(W0.a - Wm.a, Wp.a - W0.a), limiter<LIM>(W0.b - Wm.b, Wp.b - W0.b),
              limiter<LIM>(W0.c - Wm.c, Wp.c - W0.c), limiter<LIM>(W0.d - Wm.d, Wp.d - W0.d)};
}

// solver2d.hpp:25-27 with s = +1 (right/top edge) or -1 (left/bottom edge): W + (0.5*s)*dW.
__device__ __forceinline__ Q4 edge(const Q4& W, const Q4& dW, double s) {
    double h = 0.5 * s;
    return Q4{W.a + h * dW.a, W.b + h * dW.b, W.c + h * dW.c, W.d + h * dW.d};
}

// riemann2d.hpp:11-15, on two face sides (conserved state, its primitive state and sound speed)
__device__ __forceinline__ Q4 rusanov_flux(const FaceSide& L, const FaceSide& R) {
    const Q4 &UL = L.U, &WL = L.W, &UR = R.U, &WR = R.W;
    double s_max = smax(fabs(WL.b) + L.a, fabs(WR.b) + R.a);
    Q4 FL = flux_x(UL, WL), FR = flux_x(UR, WR);
    double h = 0.5 * s_max;
    return Q4{0.5 * (FL.a + FR.a) - h * (UR.a - UL.a), 0.5 * (FL.b + FR.b) - h * (UR.b - UL.b),
              0.5 * (FL.c + FR.c) - h * (UR.c - UL.c), 0.5 * (FL.d + FR.d) - h * (UR.d - UL.d)};
}

// riemann2d.hpp:27-39 (Davis wave speeds, Toro eq. 10.39 star state riemann2d.hpp:18-24).
// The reference evaluates only the branch it returns; here the upwind side is selected first
// (left when 0 <= SL or 0 <= S_star, as its first two branches are) and the star state is evaluated
// once for that side, so that all lanes of a warp run one code path.  Every branch returns the same
// expression on the same inputs as the reference, hence bit-identical results.
__device__ __forceinline__ Q4 hllc_flux(const FaceSide& L, const FaceSide& R) {
    const Q4 &UL = L.U, &WL = L.W, &UR = R.U, &WR = R.W;
    const double aL = L.a, aR = R.a;
    double SL = smin(WL.b - aL, WR.b - aR);
    double SR = smax(WL.b + aL, WR.b + aR);
    double S_star = div_z(WR.d - WL.d + WL.a * WL.b * (SL - WL.b) - WR.a * WR.b * (SR - WR.b),
                          WL.a * (SL - WL.b) - WR.a * (SR - WR.b));
    const bool left = (0.0 <= SL) || (0.0 <= S_star);
    const Q4& U = left ? UL : UR;
    const Q4& W = left ? WL : WR;
    const double S = left ? SL : SR;
    Q4 F = flux_x(U, W);
    if (0.0 <= SL || !(left || 0.0 <= SR)) return F;   // pure upwind: F(UL) if 0<=SL, F(UR) if SR<0
    double factor = div_z(W.a * (S - W.b), S - S_star);
#ifndef FV_TOLERANCE_BUILD
    const double e_rho = fdiv(U.d, W.a);
#else
    const double e_rho = U.d * (left ? L.r : R.r);  // E / rho with the side's reciprocal
#endif
    Q4 st{factor, factor * S_star, factor * W.c,
          factor * (e_rho + (S_star - W.b) * (S_star + fdiv(W.d, W.a * (S - W.b))))};
    return Q4{F.a + S * (st.a - U.a), F.b + S * (st.b - U.b), F.c + S * (st.c - U.c), F.d + S * (st.d - U.d)};
}

// Flux scheme chosen at compile time (one kernel instance per scheme), on two face sides.
template <int FLUX>
__device__ __forceinline__ Q4 face_flux(const FaceSide& L, const FaceSide& R) {
    if constexpr (FLUX == FLUX_HLLC) return hllc_flux(L, R);
    else return rusanov_flux(L, R);
}

// A face side from a conserved state alone: the FluxFn interface (riemann2d.hpp:8), which
// recomputes the primitive state and sound speed from U.
__device__ __forceinline__ FaceSide side_of(const Q4& U) {
    const Q4 W = to_primitive(U);
#ifndef FV_TOLERANCE_BUILD
    return FaceSide{U, W, sound_speed(W), 0.0};
#else
    const double r = recip(U.a);
    return FaceSide{U, W, sqrt(GAMMA * W.d * r), r};
#endif
}
template <int FLUX>
__device__ __forceinline__ Q4 face_flux(const Q4& UL, const Q4& UR) {
    return face_flux<FLUX>(side_of(UL), side_of(UR));
}

// The same face seen by a y-face: the momentum components swapped (flux_y_face, riemann2d.hpp:42-44).
__device__ __forceinline__ FaceSide swapped(const FaceSide& f) {
    return FaceSide{Q4{f.U.a, f.U.c, f.U.b, f.U.d}, Q4{f.W.a, f.W.c, f.W.b, f.W.d}, f.a, f.r};
}

// state2d.hpp:39
__device__ __forceinline__ Q4 swap_xy(const Q4& U) { return Q4{U.a, U.c, U.b, U.d}; }

// Ghost-cell source index for column/row g of an axis of n physical cells (grid2d.hpp:43-66):
// periodic ghosts copy the opposite end (modulo n), transmissive ghosts copy the nearest physical cell.
// Any g is mapped to a valid index, so tiles that overhang the grid read in-bounds memory.
__device__ __forceinline__ int bc_index(int g, int n, int bc) {
    if (bc == BC_PERIODIC) {
        int m = g % n;
        return m < 0 ? m + n : m;
    }
    return g < 0 ? 0 : (g >= n ? n - 1 : g);
}

}  // namespace fv
