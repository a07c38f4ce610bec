/* Parameter block shared by the oracle drivers of the reference solvers
 * (oracle/ref_euler_hook.cpp, oracle/ref_allaire_hook.cpp) and by the plain-C
 * restatement (oracle/cfd_oracle.c).  TEST INFRASTRUCTURE ONLY.
 *
 * Field meanings follow the reference's sim_info (headers/sim_info.hpp:16-36)
 * and the EOS parameter structs (headers/stiffened_gas_eos.hpp:20-63).
 */
#ifndef CFD_ORACLE_REF_COMMON_H
#define CFD_ORACLE_REF_COMMON_H

#ifdef __cplusplus
extern "C" {
#endif

enum { REF_LIM_MINMOD = 0, REF_LIM_VANLEER = 1, REF_LIM_MC = 2, REF_LIM_UNLIMITED = 3 };
enum { REF_FLUX_MUSCL = 0, REF_FLUX_GODUNOV = 1 };
enum { REF_SPLIT_NAIVE = 0, REF_SPLIT_STRANG = 1 };
enum { REF_WS_DAVIS = 0, REF_WS_PVRS = 1 };

typedef struct ref_params {
    int nx, ny;             /* interior cells in x (columns) and y (rows) */
    double x0, y0, dx, dy;  /* domain origin and spacing */
    double gamma1, pinf1;   /* material 1 (the only one for Euler) */
    double gamma2, pinf2;   /* material 2 (Allaire) */
    int bc[4];              /* L, R, B, T: 0 transmissive, 1 reflective */
    double cfl, T;          /* CFL number and end time */
    int limiter;            /* REF_LIM_* */
    int flux_solver;        /* REF_FLUX_* */
    int splitting;          /* REF_SPLIT_* */
    int wavespeed;          /* REF_WS_* (Allaire HLLC) */
    double z_min;           /* Allaire volume-fraction clip [z_min, 1-z_min] */
    int fix_dy_halfstep;    /* 1: use dy in the y-sweep half-step */
} ref_params;

#ifdef __cplusplus
}
#endif
#endif
