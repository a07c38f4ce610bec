// Device physics for the split finite-volume update, plain FP64 form.
//
// Every function restates a reference function (paths relative to the
// reference project; E/ = euler_equations/euler_simulation_code/, A/ =
// allaire_2d/) with the same expression tree, operation by operation.  This
// file is compiled with --fmad=false, so no multiply-add is contracted and
// results are bit-identical to the reference's x86-64 build.  Where a value is
// computed twice by the reference from identical inputs with identical
// operations, it is computed once here and reused; that cannot change a bit.
#pragma once

#include <cstdint>

namespace cfd {

enum { MODEL_EULER = 0, MODEL_ALLAIRE = 1 };
enum { LIM_MINMOD = 0, LIM_VANLEER = 1, LIM_MC = 2, LIM_UNLIMITED = 3 };
enum { WS_DAVIS = 0, WS_PVRS = 1 };

// Material parameters.  gm1_* = gamma - 1 and gp1 = gamma1 * pinf1 are formed
// with the same single operation the reference performs inline.
struct Eos {
    double g1, p1, g2, p2;
    double gm1_1, gm1_2, gp1;
};

template <int MODEL> struct ModelTraits;
template <> struct ModelTraits<MODEL_EULER> {
    static constexpr int NV = 4, IM = 1, IT = 2, IE = 3;
};
template <> struct ModelTraits<MODEL_ALLAIRE> {
    static constexpr int NV = 6, IM = 2, IT = 3, IE = 4;
};

// std::min / std::max argument order (first argument on ties and NaN).
__device__ __forceinline__ double smin(double a, double b) { return (b < a) ? b : a; }
__device__ __forceinline__ double smax(double a, double b) { return (a < b) ? b : a; }

// ------------------------------------------------------------------ EOS ---
// E/headers/stiffened_gas_eos.hpp:68-81
__device__ __forceinline__ double sg_pressure(const Eos& q, double e, double rho) {
    return ((q.gm1_1 * rho) * e) - q.gp1;
}
__device__ __forceinline__ double sg_specific_ie(const Eos& q, double p, double rho) {
    return (p + q.gp1) / (q.gm1_1 * rho);
}
__device__ __forceinline__ double sg_soundspeed(const Eos& q, double p, double rho) {
    return sqrt((q.g1 * (p + q.p1)) / rho);
}

// A/headers/mixturemodel.hpp:20-22 (repeated in every mixture function): the
// mixture coefficients eps(z) and k(z).  A term whose stiffness pinf is 0
// gives an exact (signed) zero numerator, and a zero divided by the positive
// gamma-1 is that same zero, so the division is skipped for it.
struct Mix {
    double eps, k;
};
__device__ __forceinline__ Mix mix_coeffs(const Eos& q, double z) {
    Mix m;
    double omz = 1.0 - z;
    m.eps = z / q.gm1_1 + omz / q.gm1_2;
    double t1 = (z * q.g1) * q.p1;
    if (q.p1 != 0.0) t1 = t1 / q.gm1_1;
    double t2 = (omz * q.g2) * q.p2;
    if (q.p2 != 0.0) t2 = t2 / q.gm1_2;
    double num = t1 + t2;
    m.k = (num == 0.0 && m.eps > 0.0) ? num : num / m.eps;
    return m;
}
// A/headers/mixturemodel.hpp:18-24, 26-32, 34-40, 42-52
__device__ __forceinline__ double mix_pressure(const Mix& m, double rho, double e) {
    return ((rho * e) / m.eps) - m.k;
}
__device__ __forceinline__ double mix_specific_ie(const Mix& m, double rho, double p) {
    return ((p + m.k) * m.eps) / rho;
}
__device__ __forceinline__ double mix_soundspeed(const Mix& m, double rho, double p) {
    return sqrt((m.k + p * ((1.0 / m.eps) + 1.0)) / rho);
}
__device__ __forceinline__ double mix_shock_speed_jump(const Mix& m, double p, double rho,
                                                       double p_star) {
    double p_avg = 0.5 * (p_star + p);
    return sqrt(((p_star + m.k) + (p_avg / m.eps)) / rho);
}

// ------------------------------------------------------- cons <-> prim ---
// Primitive state with the intermediates the callers reuse.
template <int MODEL> struct Prim {
    double W[ModelTraits<MODEL>::NV];
    double e;    // specific internal energy as computed by the conversion
    double rho;  // total density
    Mix mix;     // Allaire only: coefficients of z = W[5]
};

// E/headers/misc_euler.hpp:63-79 / A/headers/misc.hpp:130-147
template <int MODEL>
__device__ __forceinline__ void cons_to_prim(const Eos& q, const double* U, Prim<MODEL>& P) {
    if constexpr (MODEL == MODEL_EULER) {
        double rho = U[0];
        double u = U[1] / rho;
        double v = U[2] / rho;
        double e = (U[3] / rho) - (0.5 * ((u * u) + (v * v)));
        P.W[0] = rho;
        P.W[1] = u;
        P.W[2] = v;
        P.W[3] = sg_pressure(q, e, rho);
        P.e = e;
        P.rho = rho;
    } else {
        double rho = U[0] + U[1];
        double u = U[2] / rho;
        double v = U[3] / rho;
        double e = (U[4] / rho) - (0.5 * ((u * u) + (v * v)));
        P.mix = mix_coeffs(q, U[5]);
        P.W[0] = U[0];
        P.W[1] = U[1];
        P.W[2] = u;
        P.W[3] = v;
        P.W[4] = mix_pressure(P.mix, rho, e);
        P.W[5] = U[5];
        P.e = e;
        P.rho = rho;
    }
}

// E/headers/misc_euler.hpp:82-97 / A/headers/misc.hpp:149-163.
// Returns the specific internal energy it used through e_out.
template <int MODEL>
__device__ __forceinline__ void prim_to_cons(const Eos& q, const double* W, double* U,
                                             double& e_out) {
    if constexpr (MODEL == MODEL_EULER) {
        double rho = W[0], u = W[1], v = W[2], p = W[3];
        double e = sg_specific_ie(q, p, rho);
        U[0] = rho;
        U[1] = rho * u;
        U[2] = rho * v;
        U[3] = (rho * e) + ((0.5 * rho) * ((u * u) + (v * v)));
        e_out = e;
    } else {
        double rho = W[0] + W[1];
        Mix m = mix_coeffs(q, W[5]);
        double e = mix_specific_ie(m, rho, W[4]);
        U[0] = W[0];
        U[1] = W[1];
        U[2] = rho * W[2];
        U[3] = rho * W[3];
        U[4] = (rho * e) + ((0.5 * rho) * ((W[2] * W[2]) + (W[3] * W[3])));
        U[5] = W[5];
        e_out = e;
    }
}

// Exact physicality test on a conserved state:
// E/headers/misc_euler.hpp:123-131, A/headers/misc.hpp:228-237.
template <int MODEL> __device__ __forceinline__ bool is_physical_exact(const double* U) {
    if constexpr (MODEL == MODEL_EULER) {
        double rho = U[0];
        double u = U[1] / rho;
        double v = U[2] / rho;
        double e = (U[3] / rho) - (0.5 * ((u * u) + (v * v)));
        return rho >= 0.0 && e >= 0.0;
    } else {
        double rho = U[0] + U[1];
        double u = U[2] / rho;
        double v = U[3] / rho;
        double e = (U[4] / rho) - (0.5 * ((u * u) + (v * v)));
        double z = U[5];
        return U[0] >= 0.0 && U[1] >= 0.0 && e >= 0.0 && z >= 0.0 && z <= 1.0;
    }
}

// Physicality test of U = prim_to_cons(W) given the specific energy e that
// prim_to_cons derived from W.  The reference recomputes e from U (three
// divisions); the recomputed value differs from e by a few ulps of
// (e + |u|^2/2), so when e clears that band by a wide margin (1e-13 relative,
// ~450 ulps) the exact test cannot fail and is skipped.  Otherwise the exact
// reference expression decides.
template <int MODEL>
__device__ __forceinline__ bool is_physical_from_prim(const double* U, const double* W, double e) {
    if constexpr (MODEL == MODEL_EULER) {
        double ke = 0.5 * ((W[1] * W[1]) + (W[2] * W[2]));
        if (W[0] > 0.0 && e > 1e-13 * (e + ke)) return true;
        return is_physical_exact<MODEL>(U);
    } else {
        double ke = 0.5 * ((W[2] * W[2]) + (W[3] * W[3]));
        if (U[0] >= 0.0 && U[1] >= 0.0 && U[5] >= 0.0 && U[5] <= 1.0 && (U[0] + U[1]) > 0.0 &&
            e > 1e-13 * (e + ke))
            return true;
        return is_physical_exact<MODEL>(U);
    }
}

// A/headers/misc.hpp:251-266: the non-const overload snaps near-zero partial
// densities and near-0/1 volume fractions, then tests.  Returns whether a
// value changed through `changed`.
__device__ __forceinline__ void snap_allaire(double* U, bool& changed) {
    changed = false;
    if (fabs(U[0]) < 1e-12) { changed |= (U[0] != 0.0); U[0] = 0.0; }
    if (fabs(U[1]) < 1e-12) { changed |= (U[1] != 0.0); U[1] = 0.0; }
    if (fabs(U[5]) < 1e-12) U[5] = 0.0;
    if (fabs(U[5] - 1.0) < 1e-12) U[5] = 1.0;
}

// The checks inside MUSCL-Hancock on a freshly converted state: the const
// overload for Euler (E/headers/flux_solver_MUSCLhancock.hpp:180,212) and the
// snapping overload for Allaire (A/headers/flux_solver_MUSCLhancock.hpp:324,356),
// whose snapped values are what the Riemann solver then receives.
template <int MODEL>
__device__ __forceinline__ bool muscl_check(double* U, const double* W, double e) {
    if constexpr (MODEL == MODEL_EULER) {
        return is_physical_from_prim<MODEL>(U, W, e);
    } else {
        bool changed;
        snap_allaire(U, changed);
        if (changed) return is_physical_exact<MODEL>(U);
        return is_physical_from_prim<MODEL>(U, W, e);
    }
}

// ------------------------------------------------------------- limiters ---
// E/headers/flux_solver_MUSCLhancock.hpp:67-89 (minmod), :40-65 (MC, per
// component), :30-38 (unlimited); van Leer: dL*dR > 0 ? (2*dL*dR)/(dL+dR) : 0.
__device__ __forceinline__ double limit1(int lim, double a, double b) {
    switch (lim) {
        case LIM_VANLEER:
            return ((a * b) > 0.0) ? ((2.0 * a) * b) / (a + b) : 0.0;
        case LIM_MC:
            if (b >= 0.0 && a >= 0.0) return smin(0.5 * (a + b), smin(2.0 * a, 2.0 * b));
            if (b <= 0.0 && a <= 0.0) return smax(0.5 * (a + b), smax(2.0 * a, 2.0 * b));
            return 0.0;
        case LIM_UNLIMITED:
            return 0.5 * (a + b);
        default:
            return (b > 0.0) ? smax(0.0, smin(a, b)) : smin(0.0, smax(a, b));
    }
}

// Limited slopes of all components, d = limit(W - Wm, Wp - W), with the
// limiter chosen once for the cell rather than once per component (the
// arithmetic of each component is limit1's).
template <int NV>
__device__ __forceinline__ void limit_all1(int lim, const double* Wm, const double* W,
                                           const double* Wp, double* d) {
    switch (lim) {
        case LIM_VANLEER:
#pragma unroll
            for (int k = 0; k < NV; ++k) d[k] = limit1(LIM_VANLEER, W[k] - Wm[k], Wp[k] - W[k]);
            break;
        case LIM_MC:
#pragma unroll
            for (int k = 0; k < NV; ++k) d[k] = limit1(LIM_MC, W[k] - Wm[k], Wp[k] - W[k]);
            break;
        case LIM_UNLIMITED:
#pragma unroll
            for (int k = 0; k < NV; ++k) d[k] = limit1(LIM_UNLIMITED, W[k] - Wm[k], Wp[k] - W[k]);
            break;
        default:
#pragma unroll
            for (int k = 0; k < NV; ++k) d[k] = limit1(LIM_MINMOD, W[k] - Wm[k], Wp[k] - W[k]);
    }
}

// ------------------------------------------------ MUSCL-Hancock half step ---
// E/headers/flux_solver_MUSCLhancock.hpp:195-201 with the Jacobian of
// E/headers/misc_euler.hpp:102-119 (A/headers/misc.hpp:189-205 for Allaire):
//   X = ((0.5*(dt/dx)) * A(W)) * d
// Each row of A has at most two non-zero entries, so X_i is the sum of two
// products and does not depend on summation order.
template <int MODEL>
__device__ __forceinline__ void jacobian_times(const Eos& q, const Prim<MODEL>& P, const double* d,
                                               double s, double* X) {
    const double* W = P.W;
    if constexpr (MODEL == MODEL_EULER) {
        double rho = W[0], u = W[1];
        double c = sg_soundspeed(q, W[3], rho);
        double su = s * u;
        X[0] = su * d[0] + (s * rho) * d[1];
        X[1] = su * d[1] + (s * (1.0 / rho)) * d[3];
        X[2] = su * d[2];
        X[3] = (s * ((rho * c) * c)) * d[1] + su * d[3];
    } else {
        double rho = P.rho;  // W[0] + W[1], identical to the conversion's
        double c = mix_soundspeed(P.mix, rho, W[4]);
        double su = s * W[2];
        X[0] = su * d[0] + (s * W[0]) * d[2];
        X[1] = su * d[1] + (s * W[1]) * d[2];
        X[2] = su * d[2] + (s * (1.0 / rho)) * d[4];
        X[3] = su * d[3];
        X[4] = (s * ((rho * c) * c)) * d[2] + su * d[4];
        X[5] = su * d[5];
    }
}

// Zero-slope evolution used when the slope-extrapolated states of a face are
// unphysical (E/headers/flux_solver_MUSCLhancock.hpp:184-201): the slopes are
// the exact +0.0 vector, so ((s*A)*0) sums products that include at least one
// +0 per row and is +0 unless a Jacobian entry is not finite.
template <int MODEL>
__device__ __forceinline__ void zero_slope_state(const Eos& q, const Prim<MODEL>& P, double s,
                                                 bool left_side, double* Wout) {
    constexpr int NV = ModelTraits<MODEL>::NV;
    double d0[NV];
#pragma unroll
    for (int k = 0; k < NV; ++k) d0[k] = 0.0;
    double X[NV];
    jacobian_times<MODEL>(q, P, d0, s, X);
#pragma unroll
    for (int k = 0; k < NV; ++k) {
        double x = X[k] + 0.0;  // any finite sum of the row is +0 in the reference
        if (left_side) Wout[k] = (P.W[k] + 0.5 * d0[k]) - x;
        else Wout[k] = (P.W[k] - 0.5 * d0[k]) - x;
    }
}

// ----------------------------------------------------------------- HLLC ---
// State quantities the Riemann solver derives from a conserved state
// (E/headers/riemann_solver_HLLC.hpp:55-67, A/headers/riemann_solver_HLLC.hpp:54-68);
// flux_conserved_var recomputes exactly these from the same state, so they
// are shared with the physical flux.
template <int MODEL> struct RPSide {
    double rho, u, v, e, p, c;
    Mix mix;
};

template <int MODEL>
__device__ __forceinline__ void rp_side(const Eos& q, const double* U, RPSide<MODEL>& S) {
    if constexpr (MODEL == MODEL_EULER) {
        S.rho = U[0];
        S.u = U[1] / S.rho;
        S.v = U[2] / S.rho;
        S.e = (U[3] / S.rho) - (0.5 * ((S.u * S.u) + (S.v * S.v)));
        S.p = sg_pressure(q, S.e, S.rho);
        S.c = sg_soundspeed(q, S.p, S.rho);
    } else {
        S.rho = U[0] + U[1];
        S.u = U[2] / S.rho;
        S.v = U[3] / S.rho;
        S.e = (U[4] / S.rho) - (0.5 * ((S.u * S.u) + (S.v * S.v)));
        S.mix = mix_coeffs(q, U[5]);
        S.p = mix_pressure(S.mix, S.rho, S.e);
        S.c = mix_soundspeed(S.mix, S.rho, S.p);
    }
}

// flux_conserved_var (E/headers/misc_euler.hpp:20-39, A/headers/misc.hpp:31-52)
// from the u and p the Riemann solver already derived from the same state.
template <int MODEL>
__device__ __forceinline__ void physical_flux(const double* U, const RPSide<MODEL>& S, double* F) {
    if constexpr (MODEL == MODEL_EULER) {
        F[0] = U[0] * S.u;
        F[1] = (U[1] * S.u) + S.p;
        F[2] = U[2] * S.u;
        F[3] = (U[3] + S.p) * S.u;
    } else {
        F[0] = U[0] * S.u;
        F[1] = U[1] * S.u;
        F[2] = (U[2] * S.u) + S.p;
        F[3] = U[3] * S.u;
        F[4] = (U[4] + S.p) * S.u;
        F[5] = 0.0;
    }
}

// HLLC flux (E/headers/riemann_solver_HLLC.hpp:50-145,
// A/headers/riemann_solver_HLLC.hpp:49-150).  The reference blends both star
// fluxes with weights (1 +/- copysign(1,u*))/2, i.e. exactly 1 and 0; only
// the selected side is evaluated here, which equals the blend except for the
// sign of an exact-zero component.  wavespeed WS_PVRS uses the PVRS-based
// estimate restated from A/headers/riemann_solver_HLLC.hpp:84-107.
template <int MODEL>
__device__ __forceinline__ void hllc_flux(const Eos& q, int wavespeed, const double* UL,
                                          const double* UR, double* F, double& u_star) {
    using T = ModelTraits<MODEL>;
    constexpr int NV = T::NV;
    RPSide<MODEL> L, R;
    rp_side<MODEL>(q, UL, L);
    rp_side<MODEL>(q, UR, R);
    double SL, SR;
    if (MODEL == MODEL_ALLAIRE && wavespeed == WS_PVRS) {
        double rho_avg = 0.5 * (L.rho + R.rho);
        double c_avg = 0.5 * (L.c + R.c);
        double ppv = smax(0.0, (0.5 * (L.p + R.p)) + (((0.5 * (L.u - R.u)) * rho_avg) * c_avg));
        SL = (ppv > L.p) ? L.u - mix_shock_speed_jump(L.mix, L.p, L.rho, ppv) : L.u - L.c;
        SR = (ppv > R.p) ? R.u + mix_shock_speed_jump(R.mix, R.p, R.rho, ppv) : R.u + R.c;
    } else {
        double u_avg = 0.5 * (L.u + R.u);
        double c_avg = 0.5 * (L.c + R.c);
        SL = smin(u_avg - c_avg, L.u - L.c);
        SR = smax(u_avg + c_avg, R.u + R.c);
    }
    double dSL = SL - L.u, dSR = SR - R.u;
    double us = (((R.p - L.p) + ((L.rho * L.u) * dSL)) - ((R.rho * R.u) * dSR)) /
                ((L.rho * dSL) - (R.rho * dSR));
    u_star = us;
    bool left = !signbit(us);  // copysign(1.0, u*) == +1
    // The unselected side enters the reference's blend multiplied by exactly
    // 0, which only matters when it is not finite (0 * inf = NaN).  Its star
    // factor dS / (S - u*) and p / dS are the only terms that can blow up
    // from finite states; when either denominator is tiny the full blend is
    // evaluated as the reference does.
    double dS_o = left ? dSR : dSL;
    double den_o = (left ? SR : SL) - us;
    bool risky = !(fabs(dS_o) > 1e-200) || !(fabs(den_o) > 1e-200 * fabs(dS_o));
    if (risky) {
        double fL = dSL / (SL - us), fR = dSR / (SR - us);
        double sL[NV], sR[NV], FL[NV], FR[NV];
#pragma unroll
        for (int k = 0; k < NV; ++k) {
            sL[k] = fL * UL[k];
            sR[k] = fR * UR[k];
        }
        sL[T::IM] = (fL * L.rho) * us;
        sR[T::IM] = (fR * R.rho) * us;
        sL[T::IE] = fL * (UL[T::IE] + ((us - L.u) * ((L.rho * us) + (L.p / dSL))));
        sR[T::IE] = fR * (UR[T::IE] + ((us - R.u) * ((R.rho * us) + (R.p / dSR))));
        physical_flux<MODEL>(UL, L, FL);
        physical_flux<MODEL>(UR, R, FR);
        if constexpr (MODEL == MODEL_ALLAIRE) {
            sL[5] = 0.0;
            sR[5] = 0.0;
        }
        double cs = copysign(1.0, us);
        double a = (1.0 + cs) / 2.0, b = (1.0 - cs) / 2.0;
        double mSL = smin(0.0, SL), MSR = smax(0.0, SR);
#pragma unroll
        for (int k = 0; k < NV; ++k)
            F[k] = (a * (FL[k] + (mSL * (sL[k] - UL[k])))) + (b * (FR[k] + (MSR * (sR[k] - UR[k]))));
        if constexpr (MODEL == MODEL_ALLAIRE) F[5] = 0.0;
        return;
    }
    const double* U = left ? UL : UR;
    const RPSide<MODEL>& S = left ? L : R;
    double Sk = left ? SL : SR;
    double dS = left ? dSL : dSR;
    double fac = dS / (Sk - us);
    double wave = left ? smin(0.0, SL) : smax(0.0, SR);
    double Us[NV];
#pragma unroll
    for (int k = 0; k < NV; ++k) Us[k] = fac * U[k];
    Us[T::IM] = (fac * S.rho) * us;
    Us[T::IE] = fac * (U[T::IE] + ((us - S.u) * ((S.rho * us) + (S.p / dS))));
    if constexpr (MODEL == MODEL_ALLAIRE) Us[5] = 0.0;
    double Fp[NV];
    physical_flux<MODEL>(U, S, Fp);
#pragma unroll
    for (int k = 0; k < NV; ++k) F[k] = Fp[k] + (wave * (Us[k] - U[k]));
    if constexpr (MODEL == MODEL_ALLAIRE) F[5] = 0.0;
}

// Allaire z-update (A/headers/zupdate.hpp:44-49 upwind, :62-67 second order);
// z_min > 0 clips to [z_min, 1 - z_min] instead of [0, 1].
__device__ __forceinline__ double z_update(bool godunov, double k, double zL, double z, double zR,
                                           double usL, double usR, double zsL, double zsR,
                                           double z_min) {
    double nz;
    if (godunov)
        nz = z - (k * (((zR - z) * smin(0.0, usR)) + ((z - zL) * smax(0.0, usL))));
    else
        nz = z - (k * (((usR * zsR) - (usL * zsL)) - (z * (usR - usL))));
    if (z_min > 0.0) return smax(smin(1.0 - z_min, nz), z_min);
    return smax(smin(1.0, nz), 0.0);
}

}  // namespace cfd
