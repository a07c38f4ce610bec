/* cfdgpu_host.h -- host-side hooks of the cfdgpu library: initial conditions,
 * settingsfile.txt parsing and the reference's output formats, in the
 * reference's ghosted AoS grid layout (see cfdgpu.h).  C ABI, no device code.
 */
#ifndef CFDGPU_HOST_H
#define CFDGPU_HOST_H

#include <stddef.h>
#include <stdint.h>

#include "cfdgpu.h"

#ifdef __cplusplus
extern "C" {
#endif

/* Seeded workload recipes (new initial conditions, not in the reference). */
enum {
    CFD_RECIPE_FOUR_QUADRANT = 1,        /* 2D Riemann problem, gamma 1.4, [0,1]^2, t = 0.3 */
    CFD_RECIPE_SHOCK_BUBBLES = 2,        /* Mach-2 shock + seeded density bubbles, [0,1]^2 */
    CFD_RECIPE_WATER_SHOCK_AIR_BUBBLE = 3 /* Allaire: 1e9 Pa water shock on an air bubble, [0,2]x[0,1] */
};

/* Doubles in a ghosted AoS grid for cfg: the size of the reference's
 * gridtype (sourcecode/euler_io.cpp:494). */
int cfd_ic_grid_elems(const cfd_config* cfg, size_t* elems);

/* set_parameters of a named reference test case
 * (E/sourcecode/euler_io.cpp:13-234, A/sourcecode/allaire_diffuse_io.cpp:13-310):
 * fills domain, materials, boundary conditions and T; solver options get the
 * reference defaults (MUSCL-Hancock, minmod, HLLC, naive splitting, CFL 0.5). */
int cfd_case_config(int model, const char* test_case, int nx, int ny, int flux_solver,
                    cfd_config* cfg);

/* set_ICs of a named reference test case into `grid` (ghosted AoS, ghosts
 * included as the reference fills them; E/sourcecode/euler_io.cpp:436-731,
 * A/sourcecode/allaire_diffuse_io.cpp:402-990).  `seed` is used only by the
 * Euler case "internet", which the reference seeds from std::random_device. */
int cfd_case_ic(const cfd_config* cfg, const char* test_case, uint64_t seed, double* grid);

/* Configuration and initial condition of a seeded recipe.  No counterpart in
 * the reference: these are the benchmark workloads' initial conditions. */
int cfd_recipe_config(int recipe, int nx, int ny, cfd_config* cfg);
int cfd_recipe_ic(const cfd_config* cfg, int recipe, uint64_t seed, int nbubbles, double* grid);

/* settingsfile.txt (headers/settings_file.hpp:35-71): key/value lines; the
 * reference keys plus optional extensions (precision, steps, limiter,
 * wavespeed, alpha_clip, fix_dy_halfstep, seed, nbubbles).  Unknown keys are
 * ignored, as in the reference. */
typedef struct cfd_settings {
    int Nx, Ny;
    double CFL;
    char splitting_scheme[64];
    char test_case[128];
    int output_freq;
    char outputpath[512];
    char basename[768];
    char flux_solver[32];
    char riemann_solver[32];
    char problem[32];
    /* extensions */
    char precision[16];
    char limiter[16];
    char wavespeed[16];
    int steps;          /* 0: run to T */
    double alpha_clip;  /* z_min */
    int fix_dy_halfstep;
    uint64_t seed;
    int nbubbles;
} cfd_settings;

/* Parses a settings file (headers/settings_file.hpp:35-71, basename as :69). */
int cfd_read_settings(const char* path, cfd_settings* out);

/* Fills a solver configuration (and the initial grid when grid != NULL) from
 * settings: a reference test case name or a recipe name
 * ("four_quadrant", "shock_bubbles", "water_shock_air_bubble").  Replaces
 * set_ICs' reading of the settings (E/sourcecode/euler_io.cpp:436-461) and
 * set_splitting_scheme (headers/splitting_scheme.hpp:125-143). */
int cfd_settings_config(const cfd_settings* s, cfd_config* cfg);
int cfd_settings_ic(const cfd_settings* s, const cfd_config* cfg, double* grid);

/* Output writers in the reference formats, from a ghosted AoS grid:
 *   <basename>-state-<t>.dat       (E/sourcecode/euler_io.cpp:1188-1216,
 *                                   A/sourcecode/allaire_diffuse_io.cpp:1155-1186)
 *   <basename>-schlieren-<t>.dat   (E: :1142-1185)
 * with <t> formatted like std::to_string(double). */
int cfd_write_state(const cfd_config* cfg, const double* grid, const char* basename, double t);
int cfd_write_schlieren(const cfd_config* cfg, const double* grid, const char* basename, double t);
/* The schlieren file from a field of |grad rho| values (nx*ny, bottom row
 * first; cfd_schlieren computes it on the device): normalised by its
 * maximum and written exactly as cfd_write_schlieren writes it. */
int cfd_write_schlieren_field(const cfd_config* cfg, const double* field, const char* basename,
                              double t);
/* Allaire lineouts <basename>-lineoutx-<n>.dat and -lineouty-<n>.dat: row
 * Ny/2 and column Nx/2 of the ghosted grid, ghost cells included
 * (A/sourcecode/allaire_diffuse_io.cpp:1188-1232). */
int cfd_write_lineout(const cfd_config* cfg, const double* grid, const char* basename, int n);
/* <basename>-masschange.dat from per-step (t, mass1, mass2) records
 * (E: :1219-1233, A: :1235-1249). */
int cfd_write_masschange(const cfd_config* cfg, const char* basename, int nrec, const double* t,
                         const double* mass1, const double* mass2);

#ifdef __cplusplus
}
#endif
#endif
