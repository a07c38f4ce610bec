/* Plain-C restatement of cfd-art's split finite-volume update (Euler and
 * Allaire five-equation models).  TEST INFRASTRUCTURE ONLY -- the checker for
 * the CUDA path, never linked into the shipped library.
 *
 * Every function below restates one reference function and cites it.  Paths:
 *   E/ = euler_equations/euler_simulation_code/
 *   A/ = allaire_2d/
 * The arithmetic follows the reference's expression trees operation by
 * operation (compiled with -ffp-contract=off), so results are bit-identical to
 * the reference binary built in oracle/_ref (checked by the tests).  The
 * hooks for features the reference lacks (van Leer, PVRS wave speeds, the
 * volume-fraction clip, the dy half-step fix) restate the same hooks as
 * oracle/ref_*_hook.cpp.
 */
#include "cfd_oracle.h"

#include <math.h>
#include <stdlib.h>
#include <string.h>

#define MAXV 6

/* std::min / std::max semantics (first argument returned on ties/NaN). */
static inline double smin(double a, double b) { return (b < a) ? b : a; }
static inline double smax(double a, double b) { return (a < b) ? b : a; }

typedef struct {
    int model, nv;
    double g1, p1, g2, p2;
} eosp;

/* ---------------------------------------------------------------- EOS --- */
/* E/headers/stiffened_gas_eos.hpp:68-81 */
static double sg_pressure(double g, double pinf, double e, double rho) {
    return (g - 1.0) * rho * e - g * pinf;
}
static double sg_specific_ie(double g, double pinf, double p, double rho) {
    return (p + g * pinf) / ((g - 1.0) * rho);
}
static double sg_soundspeed(double g, double pinf, double p, double rho) {
    return sqrt((g * (p + pinf)) / rho);
}

/* A/headers/mixturemodel.hpp:18-52 */
static void mix_eps_k(const eosp* q, double z, double* eps, double* k) {
    double e = z / (q->g1 - 1.0) + (1.0 - z) / (q->g2 - 1.0);
    *k = (z * q->g1 * q->p1 / (q->g1 - 1.0) + (1.0 - z) * q->g2 * q->p2 / (q->g2 - 1.0)) / e;
    *eps = e;
}
static double mix_pressure(const eosp* q, double rho, double e, double z) {
    double eps, k;
    mix_eps_k(q, z, &eps, &k);
    return rho * e / eps - k;
}
static double mix_specific_ie(const eosp* q, double rho, double p, double z) {
    double eps, k;
    mix_eps_k(q, z, &eps, &k);
    return (p + k) * eps / rho;
}
static double mix_soundspeed(const eosp* q, double rho, double p, double z) {
    double eps, k;
    mix_eps_k(q, z, &eps, &k);
    return sqrt((k + p * ((1.0 / eps) + 1.0)) / rho);
}
static double mix_shock_speed_jump(const eosp* q, double p, double rho, double p_star, double z) {
    double eps, k;
    mix_eps_k(q, z, &eps, &k);
    double p_avg = 0.5 * (p_star + p);
    return sqrt((p_star + k + p_avg / eps) / rho);
}

/* ------------------------------------------------------- state helpers --- */
/* E/headers/misc_euler.hpp:63-79, A/headers/misc.hpp:130-147 */
static void c2p(const eosp* q, const double* U, double* W) {
    if (q->model == ORACLE_EULER) {
        double rho = U[0];
        double u = U[1] / rho;
        double v = U[2] / rho;
        double e = U[3] / rho - 0.5 * (u * u + v * v);
        W[0] = rho;
        W[1] = u;
        W[2] = v;
        W[3] = sg_pressure(q->g1, q->p1, e, rho);
    } else {
        double rho = U[0] + U[1];
        double u = U[2] / rho;
        double v = U[3] / rho;
        double e = U[4] / rho - 0.5 * (u * u + v * v);
        double p = mix_pressure(q, rho, e, U[5]);
        W[0] = U[0];
        W[1] = U[1];
        W[2] = u;
        W[3] = v;
        W[4] = p;
        W[5] = U[5];
    }
}

/* E/headers/misc_euler.hpp:82-97, A/headers/misc.hpp:149-163 */
static void p2c(const eosp* q, const double* W, double* U) {
    if (q->model == ORACLE_EULER) {
        double rho = W[0], u = W[1], v = W[2], p = W[3];
        double e = sg_specific_ie(q->g1, q->p1, p, rho);
        U[0] = rho;
        U[1] = rho * u;
        U[2] = rho * v;
        U[3] = rho * e + 0.5 * rho * (u * u + v * v);
    } else {
        double rho = W[0] + W[1];
        double e = mix_specific_ie(q, rho, W[4], W[5]);
        U[0] = W[0];
        U[1] = W[1];
        U[2] = rho * W[2];
        U[3] = rho * W[3];
        U[4] = rho * e + 0.5 * rho * (W[2] * W[2] + W[3] * W[3]);
        U[5] = W[5];
    }
}

/* E/headers/misc_euler.hpp:123-131 and A/headers/misc.hpp:228-237 (const overload) */
static int is_phys(const eosp* q, const double* U) {
    if (q->model == ORACLE_EULER) {
        double rho = U[0];
        double u = U[1] / rho;
        double v = U[2] / rho;
        double e = U[3] / rho - 0.5 * (u * u + v * v);
        return rho >= 0.0 && e >= 0.0;
    }
    double rho = U[0] + U[1];
    double u = U[2] / rho;
    double v = U[3] / rho;
    double e = U[4] / rho - 0.5 * (u * u + v * v);
    double z = U[5];
    return U[0] >= 0.0 && U[1] >= 0.0 && e >= 0.0 && z >= 0.0 && z <= 1.0;
}

/* A/headers/misc.hpp:251-266: the non-const overload snaps near-zero partial
 * densities and near-0/1 volume fractions before testing.  The reference calls
 * it inside live assert()s and in the MUSCL-Hancock checks. */
static int is_phys_snap(const eosp* q, double* U) {
    if (fabs(U[0]) < 1e-12) U[0] = 0.0;
    if (fabs(U[1]) < 1e-12) U[1] = 0.0;
    if (fabs(U[5]) < 1e-12) U[5] = 0.0;
    if (fabs(U[5] - 1.0) < 1e-12) U[5] = 1.0;
    return is_phys(q, U);
}

/* The checks inside MUSCL-Hancock: const overload for Euler, snapping
 * overload for Allaire (UL/UR are non-const members there). */
static int muscl_check(const eosp* q, double* U) {
    return q->model == ORACLE_EULER ? is_phys(q, U) : is_phys_snap(q, U);
}

/* E/headers/misc_euler.hpp:20-39, A/headers/misc.hpp:31-52 */
static void flux_cons(const eosp* q, const double* U, double* F) {
    if (q->model == ORACLE_EULER) {
        double rho = U[0];
        double u = U[1] / rho;
        double v = U[2] / rho;
        double e = U[3] / rho - 0.5 * (u * u + v * v);
        double p = sg_pressure(q->g1, q->p1, e, rho);
        F[0] = U[0] * u;
        F[1] = U[1] * u + p;
        F[2] = U[2] * u;
        F[3] = (U[3] + p) * u;
    } else {
        double rho = U[0] + U[1];
        double u = U[2] / rho;
        double v = U[3] / rho;
        double e = U[4] / rho - 0.5 * (u * u + v * v);
        double p = mix_pressure(q, rho, e, U[5]);
        F[0] = U[0] * u;
        F[1] = U[1] * u;
        F[2] = U[2] * u + p;
        F[3] = U[3] * u;
        F[4] = (U[4] + p) * u;
        F[5] = 0.0;
    }
}

/* E/headers/misc_euler.hpp:102-119, A/headers/misc.hpp:189-205:
 * primitive-variable Jacobian, returned as a dense nv x nv matrix. */
static void jacobian(const eosp* q, const double* W, double A[MAXV][MAXV]) {
    int nv = q->nv;
    for (int i = 0; i < nv; ++i)
        for (int j = 0; j < nv; ++j) A[i][j] = 0.0;
    if (q->model == ORACLE_EULER) {
        double rho = W[0], u = W[1], p = W[3];
        double c = sg_soundspeed(q->g1, q->p1, p, rho);
        for (int i = 0; i < nv; ++i) A[i][i] = u;
        A[0][1] = rho;
        A[1][3] = 1.0 / rho;
        A[3][1] = rho * c * c;
    } else {
        double rho = W[0] + W[1];
        double c = mix_soundspeed(q, rho, W[4], W[5]);
        for (int i = 0; i < nv; ++i) A[i][i] = W[2];
        A[0][2] = W[0];
        A[1][2] = W[1];
        A[2][4] = 1.0 / rho;
        A[4][2] = rho * c * c;
    }
}

/* --------------------------------------------------------- limiters --- */
/* E/headers/flux_solver_MUSCLhancock.hpp:67-89 (minmod), :40-65 (MC, sized to
 * nv), :30-38 (unlimited); van Leer is the hook limiter
 * slope = dL*dR > 0 ? (2*dL*dR)/(dL+dR) : 0. */
static void limit(int lim, int nv, const double* dL, const double* dR, double* s) {
    for (int k = 0; k < nv; ++k) {
        double a = dL[k], b = dR[k];
        switch (lim) {
            case REF_LIM_VANLEER:
                s[k] = (a * b > 0.0) ? (2.0 * a * b) / (a + b) : 0.0;
                break;
            case REF_LIM_MC:
                if (b >= 0.0 && a >= 0.0) s[k] = smin(0.5 * (a + b), smin(2.0 * a, 2.0 * b));
                else if (b <= 0.0 && a <= 0.0) s[k] = smax(0.5 * (a + b), smax(2.0 * a, 2.0 * b));
                else s[k] = 0.0;
                break;
            case REF_LIM_UNLIMITED:
                s[k] = 0.5 * (a + b);
                break;
            default:
                if (b > 0.0) s[k] = smax(0.0, smin(a, b));
                else s[k] = smin(0.0, smax(a, b));
        }
    }
}

/* ------------------------------------------------------------- HLLC --- */
/* E/headers/riemann_solver_HLLC.hpp:50-145 and A/headers/riemann_solver_HLLC.hpp:49-150.
 * wavespeed REF_WS_PVRS replaces the Davis/Garrick estimate by the PVRS-based
 * one of the commented block A/headers/riemann_solver_HLLC.hpp:84-107. */
static void hllc(const eosp* q, int wavespeed, const double* UL, const double* UR, double* flux,
                 double* u_star_out) {
    int nv = q->nv, eu = q->model == ORACLE_EULER;
    int im = eu ? 1 : 2; /* normal momentum index */
    int it = eu ? 2 : 3; /* tangential momentum */
    int ie = eu ? 3 : 4; /* energy */
    double rhoL, uL, vL, eL, pL, cL, rhoR, uR, vR, eR, pR, cR, zL = 0.0, zR = 0.0;
    if (eu) {
        rhoL = UL[0];
        uL = UL[1] / rhoL;
        vL = UL[2] / rhoL;
        eL = UL[3] / rhoL - 0.5 * (uL * uL + vL * vL);
        pL = sg_pressure(q->g1, q->p1, eL, rhoL);
        cL = sg_soundspeed(q->g1, q->p1, pL, rhoL);
        rhoR = UR[0];
        uR = UR[1] / rhoR;
        vR = UR[2] / rhoR;
        eR = UR[3] / rhoR - 0.5 * (uR * uR + vR * vR);
        pR = sg_pressure(q->g1, q->p1, eR, rhoR);
        cR = sg_soundspeed(q->g1, q->p1, pR, rhoR);
    } else {
        zL = UL[5];
        rhoL = UL[0] + UL[1];
        uL = UL[2] / rhoL;
        vL = UL[3] / rhoL;
        eL = UL[4] / rhoL - 0.5 * (uL * uL + vL * vL);
        pL = mix_pressure(q, rhoL, eL, zL);
        cL = mix_soundspeed(q, rhoL, pL, zL);
        zR = UR[5];
        rhoR = UR[0] + UR[1];
        uR = UR[2] / rhoR;
        vR = UR[3] / rhoR;
        eR = UR[4] / rhoR - 0.5 * (uR * uR + vR * vR);
        pR = mix_pressure(q, rhoR, eR, zR);
        cR = mix_soundspeed(q, rhoR, pR, zR);
    }
    (void)vL;
    (void)vR;
    double SL, SR;
    if (wavespeed == REF_WS_PVRS && !eu) {
        double rho_avg = 0.5 * (rhoL + rhoR);
        double c_avg = 0.5 * (cL + cR);
        double ppv = smax(0.0, 0.5 * (pL + pR) + 0.5 * (uL - uR) * rho_avg * c_avg);
        SL = (ppv > pL) ? uL - mix_shock_speed_jump(q, pL, rhoL, ppv, zL) : uL - cL;
        SR = (ppv > pR) ? uR + mix_shock_speed_jump(q, pR, rhoR, ppv, zR) : uR + cR;
    } else {
        double u_avg = 0.5 * (uL + uR);
        double c_avg = 0.5 * (cL + cR);
        SL = smin(u_avg - c_avg, uL - cL);
        SR = smax(u_avg + c_avg, uR + cR);
    }
    double u_star = (pR - pL + rhoL * uL * (SL - uL) - rhoR * uR * (SR - uR)) /
                    (rhoL * (SL - uL) - rhoR * (SR - uR));
    double factorL = (SL - uL) / (SL - u_star);
    double factorR = (SR - uR) / (SR - u_star);
    *u_star_out = u_star;

    double sL[MAXV], sR[MAXV], FL[MAXV], FR[MAXV];
    for (int k = 0; k < nv; ++k) {
        sL[k] = factorL * UL[k];
        sR[k] = factorR * UR[k];
    }
    sL[im] = factorL * rhoL * u_star;
    sR[im] = factorR * rhoR * u_star;
    sL[it] = factorL * UL[it];
    sR[it] = factorR * UR[it];
    sL[ie] = factorL * (UL[ie] + (u_star - uL) * (rhoL * u_star + (pL / (SL - uL))));
    sR[ie] = factorR * (UR[ie] + (u_star - uR) * (rhoR * u_star + (pR / (SR - uR))));
    if (!eu) {
        sL[5] = 0.0;
        sR[5] = 0.0;
    }
    flux_cons(q, UL, FL);
    flux_cons(q, UR, FR);
    double cs = copysign(1.0, u_star);
    double a = (1.0 + cs) / 2.0, b = (1.0 - cs) / 2.0;
    double mSL = smin(0.0, SL), MSR = smax(0.0, SR);
    for (int k = 0; k < nv; ++k)
        flux[k] = a * (FL[k] + mSL * (sL[k] - UL[k])) + b * (FR[k] + MSR * (sR[k] - UR[k]));
    if (!eu) flux[5] = 0.0;
}

/* --------------------------------------------------- flux solvers --- */
/* MUSCL-Hancock: E/headers/flux_solver_MUSCLhancock.hpp:128-227,
 * A/headers/flux_solver_MUSCLhancock.hpp:272-376.  Godunov:
 * E/headers/flux_solver_godunov.hpp:29-36, A/headers/flux_solver_godunov.hpp:26-35. */
static void face_flux(const eosp* q, const ref_params* p, const double* st, double dt, double dx,
                      double* flux, double* u_star, double* z_star) {
    int nv = q->nv;
    if (p->flux_solver == REF_FLUX_GODUNOV) {
        hllc(q, p->wavespeed, st, st + nv, flux, u_star);
        if (q->model == ORACLE_ALLAIRE) {
            double cs = copysign(1.0, *u_star);
            *z_star = ((1.0 + cs) / 2.0) * st[5] + ((1.0 - cs) / 2.0) * st[nv + 5];
        }
        return;
    }
    const double *S0 = st, *S1 = st + nv, *S2 = st + 2 * nv, *S3 = st + 3 * nv;
    double pL[MAXV] = {0}, pR[MAXV] = {0}, w0[MAXV] = {0}, w3[MAXV] = {0};
    double dLf[MAXV] = {0}, dCf[MAXV] = {0}, dRf[MAXV] = {0};
    double delL[MAXV] = {0}, delR[MAXV] = {0}, UL[MAXV] = {0}, UR[MAXV] = {0}, tmp[MAXV] = {0};
    c2p(q, S1, pL);
    c2p(q, S2, pR);
    c2p(q, S0, w0);
    c2p(q, S3, w3);
    for (int k = 0; k < nv; ++k) {
        dLf[k] = pL[k] - w0[k];
        dCf[k] = pR[k] - pL[k];
        dRf[k] = w3[k] - pR[k];
    }
    limit(p->limiter, nv, dLf, dCf, delL);
    limit(p->limiter, nv, dCf, dRf, delR);

    /* Zero the slopes if the slope-extrapolated states are unphysical. */
    for (int k = 0; k < nv; ++k) tmp[k] = pL[k] + 0.5 * delL[k];
    p2c(q, tmp, UL);
    for (int k = 0; k < nv; ++k) tmp[k] = pR[k] - 0.5 * delR[k];
    p2c(q, tmp, UR);
    if (!(muscl_check(q, UL) && muscl_check(q, UR))) {
        for (int k = 0; k < nv; ++k) {
            delL[k] = 0.0;
            delR[k] = 0.0;
        }
    }

    /* Half-step evolution with the primitive Jacobian: W -/+ del/2 - (dt/dx)/2 A del. */
    double s = 0.5 * (dt / dx);
    double A[MAXV][MAXV], WL[MAXV], WR[MAXV];
    jacobian(q, pL, A);
    for (int i = 0; i < nv; ++i) {
        double acc = (s * A[i][0]) * delL[0];
        for (int j = 1; j < nv; ++j) acc = acc + (s * A[i][j]) * delL[j];
        WL[i] = (pL[i] + 0.5 * delL[i]) - acc;
    }
    jacobian(q, pR, A);
    for (int i = 0; i < nv; ++i) {
        double acc = (s * A[i][0]) * delR[0];
        for (int j = 1; j < nv; ++j) acc = acc + (s * A[i][j]) * delR[j];
        WR[i] = (pR[i] - 0.5 * delR[i]) - acc;
    }
    p2c(q, WL, UL);
    p2c(q, WR, UR);
    /* First-order fallback if the evolved states are unphysical. */
    if (!(muscl_check(q, UL) && muscl_check(q, UR))) {
        memcpy(UL, S1, sizeof(double) * nv);
        memcpy(UR, S2, sizeof(double) * nv);
    }
    hllc(q, p->wavespeed, UL, UR, flux, u_star);
    if (q->model == ORACLE_ALLAIRE) {
        double cs = copysign(1.0, *u_star);
        *z_star = 0.5 * (1.0 + cs) * UL[5] + 0.5 * (1.0 - cs) * UR[5];
    }
}

/* ------------------------------------------------------------ grid --- */
typedef struct {
    int nx, ny, g, rows, cols, nv;
    double* a;
} grid_t;

static inline double* cell(grid_t* G, int i, int j) {
    return G->a + ((size_t)i * G->cols + j) * G->nv;
}

/* E/sourcecode/euler_ppsweep.cpp:7-118, A/sourcecode/allaire_diffuse_ppsweep.cpp:7-113:
 * mirror copies into the edge ghost strips (corners untouched); reflective
 * walls negate the normal momentum. */
static void set_bcs(const eosp* q, const ref_params* p, grid_t* G) {
    int g = G->g, nx = G->nx, ny = G->ny, nv = G->nv;
    int mx = q->model == ORACLE_EULER ? 1 : 2, my = mx + 1;
    for (int i = g; i < ny + g; ++i)
        for (int j = 0; j < g; ++j) {
            memcpy(cell(G, i, j), cell(G, i, 2 * g - j - 1), sizeof(double) * nv);
            if (p->bc[0]) cell(G, i, j)[mx] = -cell(G, i, j)[mx];
        }
    for (int i = g; i < ny + g; ++i)
        for (int j = 0; j < g; ++j) {
            memcpy(cell(G, i, j + nx + g), cell(G, i, nx + g - 1 - j), sizeof(double) * nv);
            if (p->bc[1]) cell(G, i, j + nx + g)[mx] = -cell(G, i, j + nx + g)[mx];
        }
    for (int j = g; j < nx + g; ++j)
        for (int i = 0; i < g; ++i) {
            memcpy(cell(G, i, j), cell(G, 2 * g - i - 1, j), sizeof(double) * nv);
            if (p->bc[2]) cell(G, i, j)[my] = -cell(G, i, j)[my];
        }
    for (int j = g; j < nx + g; ++j)
        for (int i = 0; i < g; ++i) {
            memcpy(cell(G, i + ny + g, j), cell(G, ny + g - 1 - i, j), sizeof(double) * nv);
            if (p->bc[3]) cell(G, i + ny + g, j)[my] = -cell(G, i + ny + g, j)[my];
        }
}

/* E/sourcecode/euler_rowsweep.cpp:47-82 (and euler_colsweep.cpp:78-113):
 * restore rho or e from the old state when the update made them <= 1e-12. */
static void euler_fixup(const eosp* q, double* f, const double* old) {
    if (is_phys(q, f)) return;
    double rho = f[0];
    double u = f[1] / rho;
    double v = f[2] / rho;
    double e = f[3] / rho - 0.5 * (u * u + v * v);
    double rho_old = old[0];
    double u_old = old[1] / rho_old;
    double v_old = old[2] / rho_old;
    double e_old = old[3] / rho_old - 0.5 * (u_old * u_old + v_old * v_old);
    if (rho <= 1e-12) rho = rho_old;
    if (e <= 1e-12) e = e_old;
    double W[4] = {rho, u, v, sg_pressure(q->g1, q->p1, e, rho)};
    p2c(q, W, f);
}

/* A/headers/zupdate.hpp:44-49 (upwind) and :62-67 (second order), with the
 * hook clip interval [z_min, 1-z_min] (z_min = 0 is the reference). */
static double zupdate(const ref_params* p, double dx, double dt, double zL, double z, double zR,
                      double usL, double usR, double zsL, double zsR) {
    double nz;
    if (p->flux_solver == REF_FLUX_GODUNOV)
        nz = z - (dt / dx) * ((zR - z) * smin(0.0, usR) + (z - zL) * smax(0.0, usL));
    else
        nz = z - (dt / dx) * (usR * zsR - usL * zsL - z * (usR - usL));
    if (p->z_min > 0.0) return smax(smin(1.0 - p->z_min, nz), p->z_min);
    return smax(smin(1.0, nz), 0.0);
}

/* One directional sweep over a line of cells.  `line` holds len + 2g cells
 * (already rotated for the y-sweep), `out` receives the len interior cells.
 * E/sourcecode/euler_rowsweep.cpp:10-95, euler_colsweep.cpp:10-114,
 * A/sourcecode/allaire_diffuse_rowsweep.cpp:10-52, allaire_diffuse_colsweep.cpp:9-73. */
static void sweep_line(const eosp* q, const ref_params* p, const double* line, int len, int g,
                       double dt, double h_flux, double h_upd, double* out, double* fl, double* us,
                       double* zs) {
    int nv = q->nv;
    int m = 2 * g;
    for (int f = g; f < len + g + 1; ++f) {
        face_flux(q, p, line + (size_t)(f - g) * nv, dt, h_flux, fl + (size_t)f * nv, &us[f],
                  &zs[f]);
        (void)m;
    }
    for (int c = g; c < len + g; ++c) {
        double* o = out + (size_t)(c - g) * nv;
        const double* U = line + (size_t)c * nv;
        for (int k = 0; k < nv; ++k)
            o[k] = U[k] + (dt / h_upd) * (fl[(size_t)c * nv + k] - fl[(size_t)(c + 1) * nv + k]);
    }
    if (q->model == ORACLE_ALLAIRE) {
        for (int c = g; c < len + g; ++c) {
            double* o = out + (size_t)(c - g) * nv;
            o[5] = zupdate(p, h_upd, dt, line[(size_t)(c - 1) * nv + 5], line[(size_t)c * nv + 5],
                           line[(size_t)(c + 1) * nv + 5], us[c], us[c + 1], zs[c], zs[c + 1]);
            is_phys_snap(q, o); /* live assert(is_physical_state(...)) */
        }
    }
}

/* The lines of a sweep are independent (each writes only its own cells of
 * F and reads G), so they are split over OpenMP threads with per-thread
 * line buffers; the results do not depend on the thread count. */
static void x_sweep(const eosp* q, const ref_params* p, grid_t* G, grid_t* F, double dt) {
    int g = G->g, nx = G->nx, nv = G->nv;
#pragma omp parallel
    {
        double* out = malloc(sizeof(double) * nx * nv);
        double* fl = malloc(sizeof(double) * (nx + 2 * g + 1) * nv);
        double* us = calloc(nx + 2 * g + 1, sizeof(double));
        double* zs = calloc(nx + 2 * g + 1, sizeof(double));
#pragma omp for schedule(static)
        for (int i = g; i < G->ny + g; ++i) {
            sweep_line(q, p, cell(G, i, 0), nx, g, dt, p->dx, p->dx, out, fl, us, zs);
            for (int j = 0; j < nx; ++j) {
                double* f = cell(F, i, j + g);
                memcpy(f, out + (size_t)j * nv, sizeof(double) * nv);
                if (q->model == ORACLE_EULER) euler_fixup(q, f, cell(G, i, j + g));
            }
        }
        free(out);
        free(fl);
        free(us);
        free(zs);
    }
}

static void y_sweep(const eosp* q, const ref_params* p, grid_t* G, grid_t* F, double dt) {
    int g = G->g, ny = G->ny, nv = G->nv;
    int a = q->model == ORACLE_EULER ? 1 : 2, b = a + 1;
    int len = ny + 2 * g;
    double h_flux = p->fix_dy_halfstep ? p->dy : p->dx; /* reference: params.dx */
#pragma omp parallel
    {
        double* line = malloc(sizeof(double) * len * nv);
        double* out = malloc(sizeof(double) * ny * nv);
        double* fl = malloc(sizeof(double) * (len + 1) * nv);
        double* us = calloc(len + 1, sizeof(double));
        double* zs = calloc(len + 1, sizeof(double));
#pragma omp for schedule(static)
        for (int j = g; j < G->nx + g; ++j) {
            for (int i = 0; i < len; ++i) {
                double* L = line + (size_t)i * nv;
                memcpy(L, cell(G, i, j), sizeof(double) * nv);
                double t = L[a];
                L[a] = L[b];
                L[b] = -t;
            }
            sweep_line(q, p, line, ny, g, dt, h_flux, p->dy, out, fl, us, zs);
            for (int i = 0; i < ny; ++i) {
                double* f = cell(F, i + g, j);
                memcpy(f, out + (size_t)i * nv, sizeof(double) * nv);
                double t = f[a];
                f[a] = -f[b];
                f[b] = t;
                if (q->model == ORACLE_EULER) euler_fixup(q, f, cell(G, i + g, j));
            }
        }
        free(line);
        free(out);
        free(fl);
        free(us);
        free(zs);
    }
}

static void swap_grids(grid_t* G, grid_t* F) {
    double* t = G->a;
    G->a = F->a;
    F->a = t;
}

/* E/headers/splitting_scheme.hpp:37-67 (naive) and :78-122 (Strang). */
static void advance(const eosp* q, const ref_params* p, grid_t* G, grid_t* F, double dt) {
    if (p->splitting == REF_SPLIT_STRANG) {
        set_bcs(q, p, G);
        x_sweep(q, p, G, F, 0.5 * dt);
        swap_grids(G, F);
        set_bcs(q, p, G);
        y_sweep(q, p, G, F, dt);
        swap_grids(G, F);
        set_bcs(q, p, G);
        x_sweep(q, p, G, F, 0.5 * dt);
        swap_grids(G, F);
        return;
    }
    set_bcs(q, p, G);
    x_sweep(q, p, G, F, dt);
    swap_grids(G, F);
    set_bcs(q, p, G);
    y_sweep(q, p, G, F, dt);
    swap_grids(G, F);
}

static eosp make_eos(int model, const ref_params* p) {
    eosp q;
    q.model = model;
    q.nv = model == ORACLE_EULER ? 4 : 6;
    q.g1 = p->gamma1;
    q.p1 = p->pinf1;
    q.g2 = p->gamma2;
    q.p2 = p->pinf2;
    return q;
}

static double compute_dt(const eosp* q, const ref_params* p, grid_t* G, int n, double t,
                         double* mass) {
    double maxu = 0.0, maxv = 0.0, m1 = 0.0, m2 = 0.0;
    int g = G->g;
    for (int i = g; i < G->ny + g; ++i)
        for (int j = g; j < G->nx + g; ++j) {
            const double* U = cell(G, i, j);
            double rho, u, v, e, pr, c;
            if (q->model == ORACLE_EULER) {
                rho = U[0];
                u = U[1] / rho;
                v = U[2] / rho;
                e = U[3] / rho - 0.5 * (u * u + v * v);
                pr = sg_pressure(q->g1, q->p1, e, rho);
                c = sg_soundspeed(q->g1, q->p1, pr, rho);
                m1 += rho;
            } else {
                rho = U[0] + U[1];
                u = U[2] / rho;
                v = U[3] / rho;
                e = U[4] / rho - 0.5 * (u * u + v * v);
                pr = mix_pressure(q, rho, e, U[5]);
                c = mix_soundspeed(q, rho, pr, U[5]);
                m1 += U[0];
                m2 += U[1];
            }
            maxu = smax(maxu, fabs(u) + c);
            maxv = smax(maxv, fabs(v) + c);
        }
    if (mass) {
        mass[0] = m1 * p->dx * p->dy;
        mass[1] = m2 * p->dx * p->dy;
    }
    double cfl = p->cfl;
    if (n < 5) cfl = smin(cfl, 0.2);
    double dt = cfl * smin(p->dx / maxu, p->dy / maxv);
    if (t + dt > p->T) dt = p->T - t;
    return dt;
}

double oracle_compute_dt(int model, const ref_params* p, const double* grid, int n, double t,
                         double* mass_out) {
    eosp q = make_eos(model, p);
    grid_t G;
    G.nx = p->nx;
    G.ny = p->ny;
    G.g = p->flux_solver == REF_FLUX_GODUNOV ? 1 : 2;
    G.rows = G.ny + 2 * G.g;
    G.cols = G.nx + 2 * G.g;
    G.nv = q.nv;
    G.a = (double*)grid;
    return compute_dt(&q, p, &G, n, t, mass_out);
}

int oracle_run(int model, const ref_params* p, double* grid, double* future, int max_steps,
               int* n_io, double* t_io, double* dt_log) {
    eosp q = make_eos(model, p);
    grid_t G, F;
    G.nx = F.nx = p->nx;
    G.ny = F.ny = p->ny;
    G.g = F.g = p->flux_solver == REF_FLUX_GODUNOV ? 1 : 2;
    G.rows = F.rows = G.ny + 2 * G.g;
    G.cols = F.cols = G.nx + 2 * G.g;
    G.nv = F.nv = q.nv;
    size_t bytes = sizeof(double) * (size_t)G.rows * G.cols * G.nv;
    double* A = malloc(bytes);
    double* B = malloc(bytes);
    memcpy(A, grid, bytes);
    memcpy(B, future ? future : grid, bytes);
    G.a = A;
    F.a = B;
    int n = *n_io, taken = 0;
    double t = *t_io;
    while (t < p->T && taken < max_steps) {
        double dt = compute_dt(&q, p, &G, n, t, NULL);
        advance(&q, p, &G, &F, dt);
        if (dt_log) dt_log[taken] = dt;
        t += dt;
        n++;
        taken++;
        if (fabs(t - p->T) < 1e-12) t = p->T;
    }
    memcpy(grid, G.a, bytes);
    if (future) memcpy(future, F.a, bytes);
    free(A);
    free(B);
    *n_io = n;
    *t_io = t;
    return taken;
}

void oracle_face_flux(int model, const ref_params* p, const double* stencil, double dt, double dx,
                      double* flux, double* u_star, double* z_star) {
    eosp q = make_eos(model, p);
    double zs = 0.0;
    face_flux(&q, p, stencil, dt, dx, flux, u_star, &zs);
    if (z_star) *z_star = zs;
}
