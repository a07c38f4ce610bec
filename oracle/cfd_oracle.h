/* Plain-C restatement of cfd-art's dimensionally split finite-volume update.
 * TEST INFRASTRUCTURE ONLY: used by tests/, __graft_entry__.smoke() and the
 * CPU-baseline leg of bench.py as the checker, never by the shipped library.
 *
 * Grids use the reference's layout: ghosted (ny+2g) x (nx+2g) cells, row-major
 * with rows along y, each cell holding nvar doubles (4 for Euler, 6 for the
 * Allaire model), g = 2 for MUSCL-Hancock and 1 for Godunov.
 */
#ifndef CFD_ORACLE_H
#define CFD_ORACLE_H

#include "ref_common.h"

#ifdef __cplusplus
extern "C" {
#endif

enum { ORACLE_EULER = 0, ORACLE_ALLAIRE = 1 };

/* Time loop of headers/simulation.hpp:48-61 with an extra step-count stop.
 * `future` may be NULL (a copy of `grid` is then used as second buffer).
 * Returns the number of steps taken. */
int oracle_run(int model, const ref_params* p, double* grid, double* future, int max_steps,
               int* n_io, double* t_io, double* dt_log);

/* compute_dt of sourcecode/euler_timestep.cpp:7-44 (allaire_diffuse_timestep.cpp:8-48).
 * mass_out[0..1] receives the mass sums times dx*dy (Allaire: both fluids). */
double oracle_compute_dt(int model, const ref_params* p, const double* grid, int n, double t,
                         double* mass_out);

/* One face: flux_computation of the MUSCL-Hancock (or Godunov) flux solver. */
void oracle_face_flux(int model, const ref_params* p, const double* stencil, double dt, double dx,
                      double* flux, double* u_star, double* z_star);

/* Initial ghosted grid and parameters of a seeded workload recipe
 * (0 four-quadrant, 1 shock + bubbles, 2 water shock on an air bubble), equal
 * bit for bit to the library's cfd_recipe_ic (oracle_recipes.c). */
int oracle_recipe_ic(int recipe, int nx, int ny, unsigned long long seed, int nbubbles,
                     double* grid, ref_params* p_out);

#ifdef __cplusplus
}
#endif
#endif
