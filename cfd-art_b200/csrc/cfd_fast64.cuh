// Fast FP64 form of the split sweeps: batch members of precision
// CFD_PREC_FP64_FAST.
//
// The method and the reference semantics are those of the plain FP64
// sweeps (cfd_sweep.cuh and cfd_physics.cuh, which restate the reference line
// by line: E/sourcecode/euler_rowsweep.cpp:10-95, euler_colsweep.cpp:10-114,
// E/headers/flux_solver_MUSCLhancock.hpp:128-227,
// E/headers/riemann_solver_HLLC.hpp:50-145 and their A/ counterparts),
// computed for throughput instead of bit identity:
//   * multiply-adds contracted into FMAs;
//   * reciprocals and square roots from the hardware approximations
//     (PTX rcp.approx.ftz.f64, rsqrt.approx.ftz.f64) refined by one
//     Newton-Raphson / Householder step to about one ulp, and one reciprocal
//     per divisor shared by every quotient over it (1/rho of a state,
//     1/(S - u*) for both star factors, 1/eps of a mixture);
//   * the primitive Jacobian product with its zero entries dropped;
//   * face states passed to the Riemann solver as primitives (no conserved
//     round trip), with the reference's physicality tests restated on them:
//     rho > 0 and p + gamma p_inf >= 0 (Euler: e >= 0); for Allaire the
//     snapping of near-zero partial densities and near-0/1 volume fractions
//     (A/headers/misc.hpp:251-266) and then the same tests;
//   * the conservative update applied face by face as the fluxes arrive.
// It agrees with the reference to a relative L1 density error far below the
// 1e-12 bound of the plain form over the benchmarked runs (measured by the
// tests against the bit-identical form), not bit for bit.
//
// Storage: the packed planes of the mixed form (cfd_mixed.cuh) hold FP64
// values instead of (value, compensation) pairs: components 0-1 as one
// double2 in the "value" float4 plane, 2-3 as one double2 in the
// "compensation" float4 plane, and for Allaire E and z as one double each in
// the two float2 planes.  Both forms take 8 bytes per component, so a member
// needs the same memory in either.
//
// Kernels: the x sweep by warp segments (lanes hold 32 consecutive cells of
// a row, neighbours by shuffles) and the y sweep by marching strips (a lane
// walks up its column with the stencil window in registers), the two
// barrier-free forms of cfd_march.cuh, over the same tile lists.
#pragma once

#include "cfd_march.cuh"

namespace cfd {
namespace fast {

using mixed::Inst;
using mixed::MixedArgs;
using mixed::TileGeom;

// Per-tile FP64 constants held in registers.
struct DPar {
    double g1, p1, gm1, gp1;  // gamma, p_inf, gamma - 1, gamma p_inf (material 1)
    double i1, i2, c1, c2;    // 1/(g1-1), 1/(g2-1), g1 p1/(g1-1), g2 p2/(g2-1)
    int flags;
    __device__ __forceinline__ int limiter() const { return flags & 3; }
    __device__ __forceinline__ bool pvrs() const { return (flags >> 2) & 1; }
    __device__ __forceinline__ bool godunov() const { return (flags >> 3) & 1; }
};

__device__ __forceinline__ DPar load_dpar(const Inst& I) {
    DPar P;
    P.g1 = I.eos.g1;
    P.p1 = I.eos.p1;
    P.gm1 = I.eos.gm1_1;
    P.gp1 = I.eos.gp1;
    P.i1 = I.pd[0];
    P.i2 = I.pd[1];
    P.c1 = I.pd[2];
    P.c2 = I.pd[3];
    P.flags = I.flags;
    return P;
}

// 1/x: the hardware approximation refined by one cubic Newton-Raphson step,
// y (1 + e + e^2) with e = 1 - x y, which takes the approximation's relative
// error to its cube (about one ulp after rounding).
__device__ __forceinline__ double rcp(double x) {
    double y;
    asm("rcp.approx.ftz.f64 %0, %1;" : "=d"(y) : "d"(x));
    const double e = fma(-x, y, 1.0);
    return fma(y, fma(e, e, e), y);
}

// sqrt(a) = a / sqrt(a): the hardware approximation of 1/sqrt(a) refined by
// one Householder step of order 3, y (1 + e/2 + 3 e^2/8) with e = 1 - a y^2;
// 0 for a = 0 and NaN for a < 0, as sqrt gives.
__device__ __forceinline__ double sqrt_f(double a) {
    double y;
    asm("rsqrt.approx.ftz.f64 %0, %1;" : "=d"(y) : "d"(a));
    const double e = fma(-a * y, y, 1.0);
    y = fma(y * fma(0.375, e, 0.5), e, y);
    return a > 0.0 ? a * y : (a == 0.0 ? 0.0 : __longlong_as_double(0x7ff8000000000000LL));
}

__device__ __forceinline__ double dmin(double a, double b) { return (b < a) ? b : a; }
__device__ __forceinline__ double dmax(double a, double b) { return (a < b) ? b : a; }

// Primitive state of a conserved one, with the reciprocals it took:
// W = (rho, u, v, p) for Euler (E/headers/misc_euler.hpp:63-79),
// (rho1 z, rho2 (1-z), u, v, p, z) for Allaire (A/headers/misc.hpp:130-147,
// pressure A/headers/mixturemodel.hpp:18-24 as p = (rho e - eps k) / eps).
template <int MODEL>
struct Prim64 {
    double W[ModelTraits<MODEL>::NV];
    double r;   // 1/rho
    double ie;  // Allaire: 1/eps
    double kn;  // Allaire: eps k
};

template <int MODEL>
__device__ __forceinline__ void mix_eps_kn(const DPar& P, double z, double& eps, double& kn) {
    const double omz = 1.0 - z;
    eps = fma(z, P.i1, omz * P.i2);
    kn = fma(z, P.c1, omz * P.c2);
}

template <int MODEL>
__device__ __forceinline__ void c2p(const DPar& P, const double* U, Prim64<MODEL>& Q) {
    if constexpr (MODEL == MODEL_EULER) {
        Q.r = rcp(U[0]);
        const double u = U[1] * Q.r, v = U[2] * Q.r;
        const double re = fma(-0.5, fma(U[1], u, U[2] * v), U[3]);  // rho e
        Q.W[0] = U[0];
        Q.W[1] = u;
        Q.W[2] = v;
        Q.W[3] = fma(P.gm1, re, -P.gp1);
    } else {
        Q.r = rcp(U[0] + U[1]);
        const double u = U[2] * Q.r, v = U[3] * Q.r;
        const double re = fma(-0.5, fma(U[2], u, U[3] * v), U[4]);
        double eps;
        mix_eps_kn<MODEL>(P, U[5], eps, Q.kn);
        Q.ie = rcp(eps);
        Q.W[0] = U[0];
        Q.W[1] = U[1];
        Q.W[2] = u;
        Q.W[3] = v;
        Q.W[4] = (re - Q.kn) * Q.ie;
        Q.W[5] = U[5];
    }
}

// rho c^2 of a primitive state: gamma (p + p_inf) (E/headers/stiffened_gas_eos.hpp:78-81),
// (k + p (1/eps + 1)) for a mixture (A/headers/mixturemodel.hpp:34-40).
template <int MODEL>
__device__ __forceinline__ double rho_c2(const DPar& P, const double* W, double ie, double kn) {
    if constexpr (MODEL == MODEL_EULER) return P.g1 * (W[3] + P.p1);
    else return fma(kn + W[4], ie, W[4]);
}

// The physicality test of a face state (E/headers/flux_solver_MUSCLhancock.hpp:178-189,
// 212-223): rho > 0 and e >= 0; for Allaire after the snapping of the
// mutating assert, which changes the state the Riemann solver receives.
template <int MODEL>
__device__ __forceinline__ bool phys(const DPar& P, double* W) {
    if constexpr (MODEL == MODEL_EULER) {
        return W[0] > 0.0 && W[3] + P.gp1 >= 0.0;
    } else {
        if (fabs(W[0]) < 1e-12) W[0] = 0.0;
        if (fabs(W[1]) < 1e-12) W[1] = 0.0;
        if (fabs(W[5]) < 1e-12) W[5] = 0.0;
        if (fabs(W[5] - 1.0) < 1e-12) W[5] = 1.0;
        double eps, kn;
        mix_eps_kn<MODEL>(P, W[5], eps, kn);
        return W[0] >= 0.0 && W[1] >= 0.0 && W[0] + W[1] > 0.0 && W[5] >= 0.0 && W[5] <= 1.0 &&
               fma(W[4], eps, kn) >= 0.0;
    }
}

// Slope limiters (E/headers/flux_solver_MUSCLhancock.hpp:30-89; van Leer
// 2 a b / (a + b) where a b > 0).
__device__ __forceinline__ double limit(int lim, double a, double b) {
    switch (lim) {
        case LIM_VANLEER: {
            const double ab = a * b;
            return ab > 0.0 ? 2.0 * ab * rcp(a + b) : 0.0;
        }
        case LIM_MC:
            if (b >= 0.0 && a >= 0.0) return dmin(0.5 * (a + b), dmin(2.0 * a, 2.0 * b));
            if (b <= 0.0 && a <= 0.0) return dmax(0.5 * (a + b), dmax(2.0 * a, 2.0 * b));
            return 0.0;
        case LIM_UNLIMITED:
            return 0.5 * (a + b);
        default:
            return (b > 0.0) ? dmax(0.0, dmin(a, b)) : dmin(0.0, dmax(a, b));
    }
}

template <int NV>
__device__ __forceinline__ void limit_all(int lim, const double* Wm, const double* W,
                                          const double* Wp, double* d) {
    switch (lim) {
        case LIM_VANLEER:
#pragma unroll
            for (int q = 0; q < NV; ++q) d[q] = limit(LIM_VANLEER, W[q] - Wm[q], Wp[q] - W[q]);
            break;
        case LIM_MC:
#pragma unroll
            for (int q = 0; q < NV; ++q) d[q] = limit(LIM_MC, W[q] - Wm[q], Wp[q] - W[q]);
            break;
        case LIM_UNLIMITED:
#pragma unroll
            for (int q = 0; q < NV; ++q) d[q] = limit(LIM_UNLIMITED, W[q] - Wm[q], Wp[q] - W[q]);
            break;
        default:
#pragma unroll
            for (int q = 0; q < NV; ++q) d[q] = limit(LIM_MINMOD, W[q] - Wm[q], Wp[q] - W[q]);
    }
}

// Evolved face states of a cell (E/headers/flux_solver_MUSCLhancock.hpp:195-201):
// Wp/Wm = W +/- d/2 - (dt/(2 dx)) A(W) d with the primitive Jacobian of
// E/headers/misc_euler.hpp:102-119 (A/headers/misc.hpp:189-205), zero entries
// dropped; fl gets bit 0/1 for a physical slope-extrapolated high/low state
// and bit 2/3 for a physical evolved high/low state.
template <int MODEL>
__device__ __forceinline__ void face_states(const DPar& P, const Prim64<MODEL>& Q, const double* d,
                                            double s, double* Wp, double* Wm, unsigned& fl) {
    constexpr int NV = ModelTraits<MODEL>::NV;
    const double* W = Q.W;
    fl = 0;
#pragma unroll
    for (int q = 0; q < NV; ++q) Wp[q] = fma(0.5, d[q], W[q]);
    if (phys<MODEL>(P, Wp)) fl |= 1u;
#pragma unroll
    for (int q = 0; q < NV; ++q) Wm[q] = fma(-0.5, d[q], W[q]);
    if (phys<MODEL>(P, Wm)) fl |= 2u;
    double X[NV];
    const double rc2 = rho_c2<MODEL>(P, W, Q.ie, Q.kn);
    if constexpr (MODEL == MODEL_EULER) {
        const double u = W[1];
        X[0] = s * fma(u, d[0], W[0] * d[1]);
        X[1] = s * fma(u, d[1], Q.r * d[3]);
        X[2] = s * (u * d[2]);
        X[3] = s * fma(rc2, d[1], u * d[3]);
    } else {
        const double u = W[2];
        X[0] = s * fma(u, d[0], W[0] * d[2]);
        X[1] = s * fma(u, d[1], W[1] * d[2]);
        X[2] = s * fma(u, d[2], Q.r * d[4]);
        X[3] = s * (u * d[3]);
        X[4] = s * fma(rc2, d[2], u * d[4]);
        X[5] = s * (u * d[5]);
    }
#pragma unroll
    for (int q = 0; q < NV; ++q) {
        Wp[q] = fma(0.5, d[q], W[q]) - X[q];
        Wm[q] = fma(-0.5, d[q], W[q]) - X[q];
    }
    if (phys<MODEL>(P, Wp)) fl |= 4u;
    if (phys<MODEL>(P, Wm)) fl |= 8u;
}

// Sound speed of a primitive state from its own reciprocals.
template <int MODEL>
__device__ __forceinline__ double sound(const DPar& P, const double* W, double r, double ie,
                                        double kn) {
    return sqrt_f(rho_c2<MODEL>(P, W, ie, kn) * r);
}

// HLLC flux from primitive face states (E/headers/riemann_solver_HLLC.hpp:50-145,
// A/headers/riemann_solver_HLLC.hpp:49-150; PVRS wave speeds restated from its
// commented block :84-107 with A/headers/riemann_solver_PVRS.hpp:85 and
// A/headers/mixturemodel.hpp:42-52).  F[NV] = u*, F[NV + 1] = z* (Allaire,
// A/headers/flux_solver_MUSCLhancock.hpp:375).  The side is selected by the
// sign bit of u* (+0 goes left), as the reference's copysign blend does.
template <int MODEL>
__device__ __forceinline__ void hllc(const DPar& P, const double* WL, const double* WR, double* F) {
    using T = ModelTraits<MODEL>;
    constexpr int NV = T::NV;
    double rhoL, rhoR, uL, uR, pL, pR, rL, rR;
    double eL = 1.0, eR = 1.0, ieL = 1.0, ieR = 1.0, knL = 0.0, knR = 0.0;  // Allaire: eps, 1/eps, eps k
    if constexpr (MODEL == MODEL_EULER) {
        rhoL = WL[0];
        rhoR = WR[0];
        uL = WL[1];
        uR = WR[1];
        pL = WL[3];
        pR = WR[3];
    } else {
        rhoL = WL[0] + WL[1];
        rhoR = WR[0] + WR[1];
        uL = WL[2];
        uR = WR[2];
        pL = WL[4];
        pR = WR[4];
        mix_eps_kn<MODEL>(P, WL[5], eL, knL);
        mix_eps_kn<MODEL>(P, WR[5], eR, knR);
        ieL = rcp(eL);
        ieR = rcp(eR);
    }
    rL = rcp(rhoL);
    rR = rcp(rhoR);
    const double cL = sound<MODEL>(P, WL, rL, ieL, knL);
    const double cR = sound<MODEL>(P, WR, rR, ieR, knR);
    double SL, SR;
    if (MODEL == MODEL_ALLAIRE && P.pvrs()) {
        const double ppv =
            dmax(0.0, fma(0.5, pL + pR, ((0.5 * (uL - uR)) * (0.5 * (rhoL + rhoR))) * (0.5 * (cL + cR))));
        // shock_speed_jump: sqrt(((p* + k) + ((p* + p)/2)/eps) / rho)
        SL = ppv > pL ? uL - sqrt_f((fma(knL, ieL, ppv) + 0.5 * (ppv + pL) * ieL) * rL) : uL - cL;
        SR = ppv > pR ? uR + sqrt_f((fma(knR, ieR, ppv) + 0.5 * (ppv + pR) * ieR) * rR) : uR + cR;
    } else {
        const double ua = 0.5 * (uL + uR), ca = 0.5 * (cL + cR);
        SL = dmin(ua - ca, uL - cL);
        SR = dmax(ua + ca, uR + cR);
    }
    const double mL = rhoL * (SL - uL), mR = rhoR * (SR - uR);
    const double us = fma(mL, uL, pR - pL) - mR * uR;
    const double u_star = us * rcp(mL - mR);
    const bool left = !signbit(u_star);
    // per-element selects (a pointer to either side would go through local memory)
    const double rho = left ? rhoL : rhoR, u = left ? uL : uR, p = left ? pL : pR;
    const double Sk = left ? SL : SR, wave = left ? dmin(0.0, SL) : dmax(0.0, SR);
    const double q = rcp(Sk - u_star);   // 1/(S - u*)
    const double fac = (Sk - u) * q;     // (S - u)/(S - u*)
    double U[NV];
    if constexpr (MODEL == MODEL_EULER) {
        const double v = left ? WL[2] : WR[2];
        U[0] = rho;
        U[1] = rho * u;
        U[2] = rho * v;
        U[3] = fma(p + P.gp1, P.i1, (0.5 * rho) * fma(u, u, v * v));
    } else {
        const double v = left ? WL[3] : WR[3];
        const double eps = left ? eL : eR, kn = left ? knL : knR;
        U[0] = left ? WL[0] : WR[0];
        U[1] = left ? WL[1] : WR[1];
        U[2] = rho * u;
        U[3] = rho * v;
        U[4] = fma(p, eps, kn) + (0.5 * rho) * fma(u, u, v * v);  // (p + k) eps + rho |u|^2 / 2
        U[5] = left ? WL[5] : WR[5];
    }
    // star state: fac U, momentum fac rho u*, energy
    // fac (E + (u* - u)(rho u* + p/(S - u))) = fac (E + (u* - u) rho u*) + (u* - u) p / (S - u*)
    const double du = u_star - u;
    double Us[NV];
#pragma unroll
    for (int k = 0; k < NV; ++k) Us[k] = fac * U[k];
    Us[T::IM] = fac * (rho * u_star);
    Us[T::IE] = fma(fac, fma(du, rho * u_star, U[T::IE]), du * (p * q));
    double Fp[NV];
    if constexpr (MODEL == MODEL_EULER) {
        Fp[0] = U[1];
        Fp[1] = fma(U[1], u, p);
        Fp[2] = U[2] * u;
        Fp[3] = (U[3] + p) * u;
    } else {
        Fp[0] = U[0] * u;
        Fp[1] = U[1] * u;
        Fp[2] = fma(U[2], u, p);
        Fp[3] = U[3] * u;
        Fp[4] = (U[4] + p) * u;
        Fp[5] = 0.0;
    }
#pragma unroll
    for (int k = 0; k < NV; ++k) F[k] = fma(wave, Us[k] - U[k], Fp[k]);
    if constexpr (MODEL == MODEL_ALLAIRE) {
        F[5] = 0.0;
        F[NV + 1] = U[5];
    }
    F[NV] = u_star;
}

// Allaire z update (A/headers/zupdate.hpp:44-49 upwind, :62-67 second
// order), clipped to [z_min, 1 - z_min] (or [0, 1]).
__device__ __forceinline__ double z_new(bool god, double k, double zL, double z, double zR,
                                        double usL, double usR, double zsL, double zsR,
                                        double z_min) {
    double nz;
    if (god)
        nz = z - k * fma(zR - z, dmin(0.0, usR), (z - zL) * dmax(0.0, usL));
    else
        nz = z - k * (fma(usR, zsR, -usL * zsL) - z * (usR - usL));
    const double lo = z_min > 0.0 ? z_min : 0.0, hi = z_min > 0.0 ? 1.0 - z_min : 1.0;
    return dmax(dmin(hi, nz), lo);
}

// Euler: the new state has rho > 0 and rho E >= |m|^2 / 2, i.e. e >= 0.
__device__ __forceinline__ bool euler_physical(const double* N) {
    return N[0] > 0.0 && fma(N[0], N[3], -0.5 * fma(N[1], N[1], N[2] * N[2])) >= 0.0;
}

// Post-update repairs of the reference: Allaire's snapping assert on the new
// state (A/sourcecode/allaire_diffuse_rowsweep.cpp:49, misc.hpp:251-266),
// Euler's density / energy restore from the old state
// (E/sourcecode/euler_rowsweep.cpp:47-82) when rho or e of the new state is
// negative (the caller reads the old state again then; it is rare).
template <int MODEL>
__device__ __forceinline__ void repair(double* N, const double* Uold) {
    if constexpr (MODEL == MODEL_ALLAIRE) {
        if (fabs(N[0]) < 1e-12) N[0] = 0.0;
        if (fabs(N[1]) < 1e-12) N[1] = 0.0;
        if (fabs(N[5]) < 1e-12) N[5] = 0.0;
        if (fabs(N[5] - 1.0) < 1e-12) N[5] = 1.0;
    } else {
        if (euler_physical(N)) return;
        double rho = N[0];
        const double u = N[1] / rho, v = N[2] / rho;
        double e = N[3] / rho - 0.5 * (u * u + v * v);
        const double ro = Uold[0];
        const double uo = Uold[1] / ro, vo = Uold[2] / ro;
        const double eo = Uold[3] / ro - 0.5 * (uo * uo + vo * vo);
        if (rho <= 1e-12) rho = ro;
        if (e <= 1e-12) e = eo;
        // the pressure of (e, rho) taken back to conserved: rho e + rho |u|^2 / 2
        N[0] = rho;
        N[1] = rho * u;
        N[2] = rho * v;
        N[3] = rho * e + 0.5 * rho * (u * u + v * v);
    }
}

// The planes of one state buffer of an FP64 member (see the storage note),
// held in registers: the stores of a sweep go through pointers the compiler
// cannot tell apart from the member descriptor, so reading the descriptor's
// pointers again after every store would cost a global load each time.
struct Planes64 {
    double2* a;  // components 0-1
    double2* b;  // components 2-3
    double* c;   // Allaire E
    double* d;   // Allaire z
};

template <int MODEL>
__device__ __forceinline__ Planes64 planes64(const Inst& I, int buf) {
    Planes64 p;
    p.a = reinterpret_cast<double2*>(I.q4[buf][0]);
    p.b = reinterpret_cast<double2*>(I.q4[buf][1]);
    p.c = MODEL == MODEL_ALLAIRE ? reinterpret_cast<double*>(I.q2[buf][0]) : nullptr;
    p.d = MODEL == MODEL_ALLAIRE ? reinterpret_cast<double*>(I.q2[buf][1]) : nullptr;
    return p;
}

// FP64 cell at element offset `off` of a buffer that the sweep only reads.
template <int MODEL>
__device__ __forceinline__ void load64(const Planes64& P, long long off, double* U) {
    const double2 a = __ldg(P.a + off);
    const double2 b = __ldg(P.b + off);
    U[0] = a.x;
    U[1] = a.y;
    U[2] = b.x;
    U[3] = b.y;
    if constexpr (MODEL == MODEL_ALLAIRE) {
        U[4] = __ldg(P.c + off);
        U[5] = __ldg(P.d + off);
    }
}

template <int MODEL>
__device__ __forceinline__ void store64(const Planes64& P, long long off, const double* U) {
    P.a[off] = make_double2(U[0], U[1]);
    P.b[off] = make_double2(U[2], U[3]);
    if constexpr (MODEL == MODEL_ALLAIRE) {
        P.c[off] = U[4];
        P.d[off] = U[5];
    }
}

// Wave speeds |u| + c, |v| + c and the mass terms of a new (unrotated) state
// (E/sourcecode/euler_timestep.cpp:9-26, A/sourcecode/allaire_diffuse_timestep.cpp:10-29).
template <int MODEL>
__device__ __forceinline__ void speeds(const DPar& P, const double* N, double& su, double& sv,
                                       double& m1, double& m2) {
    using MT = ModelTraits<MODEL>;
    Prim64<MODEL> Q;
    c2p<MODEL>(P, N, Q);
    const double c = sound<MODEL>(P, Q.W, Q.r, Q.ie, Q.kn);
    su = fabs(Q.W[MT::IM]) + c;
    sv = fabs(Q.W[MT::IT]) + c;
    m1 = N[0];
    m2 = MODEL == MODEL_ALLAIRE ? N[1] : 0.0;
}

// ---- y sweep by marching strips ---------------------------------------------

// Rows staged ahead through shared memory: a lane copies the cells of rows
// k+1 .. k+kAhead of its column global -> shared with cp.async while it
// computes row k, so no registers are held by the loads in flight; per slot
// NU 16-byte units per lane (components 0-1, 2-3, and for Allaire E and z),
// lane-major.  Euler's ring has kAhead + 2 slots: the slot refilled at row k
// is the one read at row k - 2, so row k - 1 is still there when row k
// computes and its update starts from it there rather than from registers
// (8 fewer registers, y sweep 0.448 -> 0.421 ms at 4096^2).  Allaire, 2 CTAs
// per SM either way, measured 1.5 % slower like that; it carries row k - 1
// in registers and refills the slot read at row k - 1 (kAhead + 1 slots).
constexpr int kAhead = 3;
template <int MODEL>
__host__ __device__ constexpr bool march64_reread() {
    return MODEL == MODEL_EULER;
}
template <int MODEL>
__host__ __device__ constexpr int march64_slots() {
    return kAhead + (march64_reread<MODEL>() ? 2 : 1);
}
template <int MODEL>
__host__ __device__ constexpr int stage_units() {
    return MODEL == MODEL_ALLAIRE ? 3 : 2;
}
template <int MODEL>
__host__ __device__ constexpr int march64_smem_bytes() {
    return 4 * march64_slots<MODEL>() * stage_units<MODEL>() * 32 * 16;  // 4 warps per CTA
}

template <int N>
__device__ __forceinline__ void cp_async_wait() {
    asm volatile("cp.async.wait_group %0;\n" ::"n"(N) : "memory");
}

// Starts copying the cell at element offset `off` into slot `s` of this lane.
template <int MODEL>
__device__ __forceinline__ void stage_issue(char* stg, int s, const Planes64& P, long long off) {
    constexpr int NU = stage_units<MODEL>();
    mixed::cp_async16(stg + ((s * NU + 0) * 32) * 16, P.a + off);
    mixed::cp_async16(stg + ((s * NU + 1) * 32) * 16, P.b + off);
    if constexpr (MODEL == MODEL_ALLAIRE) {
        mixed::cp_async8(stg + ((s * NU + 2) * 32) * 16, P.c + off);
        mixed::cp_async8(stg + ((s * NU + 2) * 32) * 16 + 8, P.d + off);
    }
}

template <int MODEL>
__device__ __forceinline__ void stage_read(const char* stg, int s, double* U) {
    constexpr int NU = stage_units<MODEL>();
    const double2 a = *reinterpret_cast<const double2*>(stg + ((s * NU + 0) * 32) * 16);
    const double2 b = *reinterpret_cast<const double2*>(stg + ((s * NU + 1) * 32) * 16);
    U[0] = a.x;
    U[1] = a.y;
    U[2] = b.x;
    U[3] = b.y;
    if constexpr (MODEL == MODEL_ALLAIRE) {
        const double2 c = *reinterpret_cast<const double2*>(stg + ((s * NU + 2) * 32) * 16);
        U[4] = c.x;
        U[5] = c.y;
    }
}
// A lane walks up its column from row r0 - 2 to r1 + 1 (two halo rows at each
// end, mirrored at the domain edges as pre_sweep fills them,
// E/sourcecode/euler_ppsweep.cpp:7-118).  Loading row k completes the slope
// and face states of row k - 1, the flux at the face between rows k - 2 and
// k - 1, and the update of row k - 2.  Carried from row to row: the
// primitive states of rows k - 1 and k - 2 (and 1/rho, 1/eps of row k - 1),
// the evolved high-face state of row k - 2 and the partly updated state of
// row k - 2 (its low-face flux applied); the raw state of row k - 1 is read
// again from its staging slot (Euler) or carried (Allaire).
template <int MODEL>
__device__ __forceinline__ void march64_strip(const MixedArgs& A, const TileGeom& g) {
    using MT = ModelTraits<MODEL>;
    constexpr int NV = MT::NV;
    const int lane = threadIdx.x & 31;
    const Inst& I = A.insts[g.inst];
    const DPar P = load_dpar(I);
    DevState* st = I.st;
    const double dt = st->dt;
    const double s_half = 0.5 * (dt / (I.fix_dy ? I.dy : I.dx));  // the reference: dx (quirk)
    const double k_upd = dt / I.dy;
    const int ny = g.len, nx = g.wid;
    const int col = g.b_org + lane;
    const bool live = col < nx;
    const int c = min(col, nx - 1);
    const int r0 = g.a_org + 2;
    const int r1 = min(r0 + A.rows, ny);
    // the x sweep's output -> the current buffer
    const Planes64 pin = planes64<MODEL>(I, g.cur ^ 1), pout = planes64<MODEL>(I, g.cur);
    const long long pitch = I.pitch;
    const bool wall_lo = (P.flags >> 7) & 1, wall_hi = (P.flags >> 8) & 1;
    const bool god = P.godunov();
    const int lim = P.limiter();
    const double z_min = I.z_min;

    auto src_row = [&](int k, bool& neg) {
        neg = false;
        int r = k;
        if (k < 0) {
            r = -k - 1;
            neg = wall_lo;
        } else if (k >= ny) {
            r = 2 * ny - 1 - k;
            neg = wall_hi;
        }
        return min(max(r, 0), ny - 1);
    };

    Prim64<MODEL> Q1, Q2;          // rows k-1, k-2
    double A2[NV], Pp[NV];         // partly updated row k-2, high face of row k-2
    unsigned flp = 0;
    double usL = 0.0, zsL = 0.0;   // u*, z* at the low face of row k-2
    double z3 = 0.0;               // z of row k-3 (upwind z update)
    double rmu = 0.0, rmv = 0.0, rm1 = 0.0, rm2 = 0.0;
#pragma unroll
    for (int q = 0; q < NV; ++q) Q1.W[q] = Q2.W[q] = A2[q] = Pp[q] = 0.0;
    Q1.r = Q1.ie = Q1.kn = Q2.r = Q2.ie = Q2.kn = 0.0;

    // this lane's staging slots; rows r0-2 .. r0-3+kAhead in flight first
    extern __shared__ __align__(16) char fast_stage[];
    constexpr bool reread = march64_reread<MODEL>();
    constexpr int NS = march64_slots<MODEL>();
    double H1c[NV];  // raw row k-1 in the sweep frame (when carried)
#pragma unroll
    for (int q = 0; q < NV; ++q) H1c[q] = 0.0;
    char* stg = fast_stage + (threadIdx.x >> 5) * (NS * stage_units<MODEL>() * 32 * 16) + 16 * lane;
    bool dummy;
#pragma unroll
    for (int j = 0; j < kAhead; ++j) {
        if (r0 - 2 + j <= r1 + 1) stage_issue<MODEL>(stg, j, pin, src_row(r0 - 2 + j, dummy) * pitch + c);
        mixed::cp_async_commit();
    }
    int slot = 0;

    // Euler: unrolled by two, so that the two-row window changes roles
    // instead of being copied (y sweep 2 % faster; no change for Allaire)
#pragma unroll(MODEL == MODEL_EULER ? 2 : 1)
    for (int k = r0 - 2; k <= r1 + 1; ++k) {
        double h[NV];
        bool neg;
        src_row(k, neg);
        cp_async_wait<kAhead - 1>();  // row k has arrived
        stage_read<MODEL>(stg, slot, h);
        const int slot1 = slot == 0 ? NS - 1 : slot - 1;                   // row k - 1
        const int refill = !reread ? slot1 : slot >= 2 ? slot - 2 : slot + NS - 2;  // row k - 1 or k - 2
        if (k + kAhead <= r1 + 1)
            stage_issue<MODEL>(stg, refill, pin, src_row(k + kAhead, dummy) * pitch + c);
        mixed::cp_async_commit();
        slot = slot == NS - 1 ? 0 : slot + 1;
        // sweep frame: mirror sign, then (u, v) -> (v, -u) (E/sourcecode/euler_colsweep.cpp:22-29)
        {
            const double m = h[MT::IM], n = neg ? -h[MT::IT] : h[MT::IT];
            h[MT::IM] = n;
            h[MT::IT] = -m;
        }
        Prim64<MODEL> Q0;
        c2p<MODEL>(P, h, Q0);

        // slope and face states of row k-1
        double Pn[NV], Mn[NV];
        unsigned fln = 0;
        if (k >= r0 && !god) {
            double d[NV];
            limit_all<NV>(lim, Q2.W, Q1.W, Q0.W, d);
            face_states<MODEL>(P, Q1, d, s_half, Pn, Mn, fln);
        } else {
#pragma unroll
            for (int q = 0; q < NV; ++q) Pn[q] = Mn[q] = Q1.W[q];
        }

        if (k >= r0 + 1) {
            // flux at the face between rows k-2 and k-1
            double F[NV + 2], WL[NV], WR[NV];
            const bool second = !god && (flp & 1u) && (fln & 2u) && (flp & 4u) && (fln & 8u);
#pragma unroll
            for (int q = 0; q < NV; ++q) {
                WL[q] = second ? Pp[q] : Q2.W[q];
                WR[q] = second ? Mn[q] : Q1.W[q];
            }
            hllc<MODEL>(P, WL, WR, F);

            if (k >= r0 + 2) {  // row k-2 is complete
                const int row = k - 2;
                double N[NV];
#pragma unroll
                for (int q = 0; q < NV; ++q) N[q] = fma(-k_upd, F[q], A2[q]);
                if constexpr (MODEL == MODEL_ALLAIRE)
                    N[5] = z_new(god, k_upd, z3, A2[5], Q1.W[5], usL, F[NV], zsL, F[NV + 1], z_min);
                {  // rotate back (E/sourcecode/euler_colsweep.cpp:66-73)
                    const double t = N[MT::IM];
                    N[MT::IM] = -N[MT::IT];
                    N[MT::IT] = t;
                }
                if constexpr (MODEL == MODEL_EULER) {
                    if (!euler_physical(N)) {  // the stored old state, for the restore
                        double Uo[NV];
                        load64<MODEL>(pin, row * pitch + c, Uo);
                        repair<MODEL>(N, Uo);
                    }
                } else {
                    repair<MODEL>(N, nullptr);
                }
                if (live) {
                    store64<MODEL>(pout, row * pitch + c, N);
                    double su, sv, m1, m2;
                    speeds<MODEL>(P, N, su, sv, m1, m2);
                    rmu = dmax(rmu, su);
                    rmv = dmax(rmv, sv);
                    rm1 += m1;
                    rm2 += m2;
                }
            }
            // row k-1 takes the flux at its low face (it is updated only
            // when inside the strip, so never a mirrored row)
            double H1[NV];
            if constexpr (reread) {
                stage_read<MODEL>(stg, slot1, H1);
                const double m = H1[MT::IM];
                H1[MT::IM] = H1[MT::IT];
                H1[MT::IT] = -m;
            } else {
#pragma unroll
                for (int q = 0; q < NV; ++q) H1[q] = H1c[q];
            }
#pragma unroll
            for (int q = 0; q < NV; ++q) A2[q] = fma(k_upd, F[q], H1[q]);
            if constexpr (MODEL == MODEL_ALLAIRE) {
                A2[5] = H1[5];
                z3 = Q2.W[5];
                usL = F[NV];
                zsL = F[NV + 1];
            }
        }

        // shift the window
        Q2 = Q1;
        Q1 = Q0;
#pragma unroll
        for (int q = 0; q < NV; ++q) {
            Pp[q] = Pn[q];
            if constexpr (!reread) H1c[q] = h[q];
        }
        flp = fln;
    }

    // this strip's wave speeds and masses into its slot, then the ticket
    for (int o = 16; o > 0; o >>= 1) {
        rmu = dmax(rmu, __shfl_down_sync(0xffffffffu, rmu, o));
        rmv = dmax(rmv, __shfl_down_sync(0xffffffffu, rmv, o));
        rm1 += __shfl_down_sync(0xffffffffu, rm1, o);
        rm2 += __shfl_down_sync(0xffffffffu, rm2, o);
    }
    unsigned ticket = 0;
    if (lane == 0) {
        double* p = I.partials + 4 * g.ltile;
        p[0] = rmu;
        p[1] = rmv;
        p[2] = rm1;
        p[3] = rm2;
        __threadfence();
        ticket = atomicAdd(&st->ticket, 1u);
    }
    ticket = __shfl_sync(0xffffffffu, ticket, 0);
    if (ticket + 1u == (unsigned)I.tiles_y) {
        __threadfence();
        mixed::march_finish(st, I.partials, I.tiles_y, dt);
    }
}

// Euler bounded to 128 registers for 4 CTAs per SM: its y sweep measured
// faster than at the 3 CTAs of its unbounded register count; Allaire runs 2.
template <int MODEL>
__global__ void __launch_bounds__(128, MODEL == MODEL_EULER ? 4 : 2) fast_march_kernel(MixedArgs A) {
    const int gw = blockIdx.x * (blockDim.x >> 5) + (threadIdx.x >> 5);
    const int nw = gridDim.x * (blockDim.x >> 5);
    for (int tile = gw; tile < A.ntiles; tile += nw) {
        const TileGeom g = mixed::tile_geom<DIR_Y, mixed::kMarchMaxRows, 32>(A, tile);
        if (!g.skip) march64_strip<MODEL>(A, g);
    }
}

// ---- x sweep by warp segments -----------------------------------------------
// The 32 lanes hold 32 consecutive cells of a row (kSegCells outputs and a
// 2-cell halo at each end); neighbour values come from the adjacent lanes by
// shuffles.  A warp walks the rows of its tile (A.rows, chosen per launch).
template <int N>
__device__ __forceinline__ void shfl_up64(const double* x, double* y) {
#pragma unroll
    for (int q = 0; q < N; ++q) y[q] = __shfl_up_sync(0xffffffffu, x[q], 1);
}
template <int N>
__device__ __forceinline__ void shfl_down64(const double* x, double* y) {
#pragma unroll
    for (int q = 0; q < N; ++q) y[q] = __shfl_down_sync(0xffffffffu, x[q], 1);
}

constexpr int kSegSlots = kAhead + 1;
template <int MODEL>
__host__ __device__ constexpr int segment64_smem_bytes() {
    return 4 * kSegSlots * stage_units<MODEL>() * 32 * 16;  // 4 warps per CTA
}

template <int MODEL>
__device__ __forceinline__ void segment64_tile(const MixedArgs& A, const TileGeom& g) {
    using MT = ModelTraits<MODEL>;
    constexpr int NV = MT::NV;
    const int lane = threadIdx.x & 31;
    const Inst& I = A.insts[g.inst];
    const DPar P = load_dpar(I);
    const double dt = I.st->dt;
    const double s_half = 0.5 * (dt / I.dx);
    const double k_upd = dt / I.dx;
    const int nx = g.len, ny = g.wid;
    const Planes64 pin = planes64<MODEL>(I, g.cur), pout = planes64<MODEL>(I, g.cur ^ 1);
    const long long pitch = I.pitch;
    const bool god = P.godunov();
    const int lim = P.limiter();
    const double z_min = I.z_min;
    // this lane's column and its mirrored source (pre_sweep's fill)
    const int ga = g.a_org + lane;
    int src = ga;
    bool neg = false;
    if (ga < 0) {
        src = -ga - 1;
        neg = (P.flags >> 5) & 1;
    } else if (ga >= nx) {
        src = 2 * nx - 1 - ga;
        neg = (P.flags >> 6) & 1;
    }
    src = min(max(src, 0), nx - 1);
    const bool writer = lane >= 2 && lane < 2 + mixed::kSegCells && ga < nx;
    const int row_end = min(g.b_org + A.rows, ny);

    // rows staged kAhead ahead, the slot refilled at row r the one read at row r - 1
    extern __shared__ __align__(16) char seg64_stage[];
    char* stg = seg64_stage + (threadIdx.x >> 5) * (kSegSlots * stage_units<MODEL>() * 32 * 16) + 16 * lane;
#pragma unroll
    for (int j = 0; j < kAhead; ++j) {
        if (g.b_org + j < row_end) stage_issue<MODEL>(stg, j, pin, (g.b_org + j) * pitch + src);
        mixed::cp_async_commit();
    }
    int slot = 0;
    for (int row = g.b_org; row < row_end; ++row) {
        double h[NV];
        cp_async_wait<kAhead - 1>();  // row `row` has arrived
        stage_read<MODEL>(stg, slot, h);
        if (row + kAhead < row_end)
            stage_issue<MODEL>(stg, slot == 0 ? kSegSlots - 1 : slot - 1, pin, (row + kAhead) * pitch + src);
        mixed::cp_async_commit();
        slot = slot == kSegSlots - 1 ? 0 : slot + 1;
        if (neg) h[MT::IM] = -h[MT::IM];
        Prim64<MODEL> Q;
        c2p<MODEL>(P, h, Q);
        double Wl[NV], Wr[NV];
        shfl_up64<NV>(Q.W, Wl);
        shfl_down64<NV>(Q.W, Wr);

        // slope and face states of this cell (used by lanes 1..30)
        double Pf[NV], Mf[NV];
        unsigned fl = 0;
        if (!god) {
            double d[NV];
            limit_all<NV>(lim, Wl, Q.W, Wr, d);
            face_states<MODEL>(P, Q, d, s_half, Pf, Mf, fl);
        } else {
#pragma unroll
            for (int q = 0; q < NV; ++q) Pf[q] = Mf[q] = Q.W[q];
        }

        // HLLC at this cell's low face (between the lane below and this one)
        double F[NV + 2];
        {
            double PL[NV];
            shfl_up64<NV>(Pf, PL);
            const unsigned flL = __shfl_up_sync(0xffffffffu, fl, 1);
            const bool second = !god && (flL & 1u) && (fl & 2u) && (flL & 4u) && (fl & 8u);
            double WL[NV], WR[NV];
#pragma unroll
            for (int q = 0; q < NV; ++q) {
                WL[q] = second ? PL[q] : Wl[q];
                WR[q] = second ? Mf[q] : Q.W[q];
            }
            hllc<MODEL>(P, WL, WR, F);
        }
        double FR[NV + 2];  // Euler's update needs only the NV fluxes, not u*
        shfl_down64<MODEL == MODEL_EULER ? NV : NV + 2>(F, FR);

        // update (lanes 2 .. 2 + kSegCells - 1)
        double N[NV];
#pragma unroll
        for (int q = 0; q < NV; ++q) N[q] = fma(k_upd, F[q] - FR[q], h[q]);
        if constexpr (MODEL == MODEL_ALLAIRE)
            N[5] = z_new(god, k_upd, Wl[5], h[5], Wr[5], F[NV], FR[NV], F[NV + 1], FR[NV + 1], z_min);
        if (writer) {  // interior cells: h is the stored old state
            repair<MODEL>(N, h);
            store64<MODEL>(pout, row * pitch + ga, N);
        }
    }
}

// At least 4 CTAs per SM: Allaire bounded to 128 registers measured 25 %
// faster than at the 3 CTAs of its unbounded count; Euler (96 registers)
// runs 5.
template <int MODEL>
__global__ void __launch_bounds__(128, 4) fast_segment_x_kernel(MixedArgs A) {
    const int gw = blockIdx.x * (blockDim.x >> 5) + (threadIdx.x >> 5);
    const int nw = gridDim.x * (blockDim.x >> 5);
    for (int tile = gw; tile < A.ntiles; tile += nw) {
        const TileGeom g = mixed::tile_geom<DIR_X, mixed::kSegCells, mixed::kSegRows>(A, tile);
        if (!g.skip) segment64_tile<MODEL>(A, g);
    }
}

}  // namespace fast
}  // namespace cfd
