// Oracle driver for the reference's single-gas Euler solver.
//
// TEST INFRASTRUCTURE ONLY.  This translation unit is compiled together with
// the reference's own sources (euler_equations/euler_simulation_code/
// sourcecode/euler_{io,ppsweep,rowsweep,colsweep,timestep}.cpp and its headers)
// into oracle/_ref/libref_euler.so by oracle/Makefile.  Only the tests, the
// smoke check and bench.py's CPU-baseline / reference arm load it.
//
// What it adds around the unmodified reference code (all hooks are labelled):
//   * a C entry point that runs the reference time loop
//     (headers/simulation.hpp:36-67) on a caller-supplied ghosted grid, with a
//     step-count stop in addition to the t=T stop;
//   * slope-limiter selection.  The reference hard-wires minmod
//     (headers/flux_solver_MUSCLhancock.hpp:124) and its clone() re-creates
//     the solver with minmod, so the hook subclasses the flux solver and
//     overrides clone() to keep the chosen limiter.  van Leer is a hook
//     limiter (the reference has none); MC is restated for 4 components
//     because the reference MC hard-codes 6 (flux_solver_MUSCLhancock.hpp:46);
//   * an optional "dy in the y half-step" fix (the reference passes params.dx
//     in update_col, sourcecode/euler_colsweep.cpp:43);
//   * thin wrappers over the reference's IC builders and gnuplot writers.
#include <algorithm>
#include <cassert>
#include <cmath>
#include <cstring>
#include <fstream>
#include <functional>
#include <iostream>
#include <memory>
#include <random>
#include <sstream>
#include <string>
#include <vector>
#include <omp.h>
#include <Eigen/Dense>

// The hooks need the reference's protected/private members (limiter slot,
// IC helpers, writers).  Class layout is unaffected by access specifiers.
#define private public
#define protected public
#include "euler_problem.hpp"
#include "flux_solver_MUSCLhancock.hpp"
#include "flux_solver_godunov.hpp"
#include "riemann_solver_HLLC.hpp"
#include "misc_euler.hpp"
#include "splitting_scheme.hpp"
#include "settings_file.hpp"
#include "simulation.hpp"
#undef private
#undef protected

#include "ref_common.h"

namespace {

// HOOK: van Leer limiter, slope = dL*dR > 0 ? (2*dL*dR)/(dL+dR) : 0.
vectype vanleer_slope(const vectype& dL, const vectype& dR) {
    vectype s(dL.rows());
    for (int k = 0; k < dL.rows(); ++k) {
        if (dL(k) * dR(k) > 0.0) s(k) = (2.0 * dL(k) * dR(k)) / (dL(k) + dR(k));
        else s(k) = 0.0;
    }
    return s;
}

// HOOK: the reference MC limiter (flux_solver_MUSCLhancock.hpp:40-65) with the
// component count taken from the input instead of the hard-coded 6.
vectype mc_slope_sized(const vectype& dL, const vectype& dR) {
    vectype s(dL.rows());
    for (int k = 0; k < dL.rows(); ++k) {
        if (dR(k) >= 0.0 && dL(k) >= 0.0)
            s(k) = std::min(0.5 * (dL(k) + dR(k)), std::min(2.0 * dL(k), 2.0 * dR(k)));
        else if (dR(k) <= 0.0 && dL(k) <= 0.0)
            s(k) = std::max(0.5 * (dL(k) + dR(k)), std::max(2.0 * dL(k), 2.0 * dR(k)));
        else
            s(k) = 0.0;
    }
    return s;
}

std::function<vectype(const vectype&, const vectype&)> pick_limiter(int lim) {
    switch (lim) {
        case REF_LIM_MINMOD: return minmod_limited_slope;
        case REF_LIM_VANLEER: return vanleer_slope;
        case REF_LIM_MC: return mc_slope_sized;
        case REF_LIM_UNLIMITED: return unlimited_central_diff;
    }
    return minmod_limited_slope;
}

// HOOK: reference MUSCL-Hancock solver with a selectable limiter that survives
// clone(), and with the optional dy substitution in the column sweep.
class OracleMusclEuler : public MusclEulerEquations {
public:
    int lim;
    bool fix_dy;
    bool in_col = false;
    OracleMusclEuler(std::shared_ptr<riemann_solver_base_euler_equations> rs, sim_info p,
                     double gamma, double pinf, int lim_, bool fix_dy_)
        : MusclEulerEquations(rs, p, gamma, pinf), lim(lim_), fix_dy(fix_dy_) {
        slopelimiter = pick_limiter(lim);
    }
    void flux_computation(const std::vector<vectype>& stencil, vectype& flux, double dt, double dx,
                          double& u_star, double* p_star_ptr = nullptr,
                          double* v_star_ptr = nullptr) override {
        double h = (in_col && fix_dy) ? params.dy : dx;
        MusclEulerEquations::flux_computation(stencil, flux, dt, h, u_star, p_star_ptr, v_star_ptr);
    }
    std::shared_ptr<FluxSolverBaseEulerEquations> clone() override {
        return std::make_shared<OracleMusclEuler>(RS_ptr->clone(), params, eosparams.gamma,
                                                  eosparams.pinf, lim, fix_dy);
    }
};

// HOOK: problem whose clone keeps the hook flux solver and which marks column
// sweeps so the optional dy fix can apply.
class OracleEuler : public Euler {
public:
    OracleEuler(double gamma, double pinf, std::shared_ptr<FluxSolverBaseEulerEquations> fs)
        : Euler(gamma, pinf, fs) {}
    void update_col(const gridtype& grid, gridtype& future_grid, const sim_info& params, int j,
                    double dt, double t) override {
        OracleMusclEuler* m = dynamic_cast<OracleMusclEuler*>(fs_ptr.get());
        if (m) m->in_col = true;
        Euler::update_col(grid, future_grid, params, j, dt, t);
        if (m) m->in_col = false;
    }
    std::shared_ptr<problem_base> clone() override {
        return std::make_shared<OracleEuler>(eosparams.gamma, eosparams.pinf, fs_ptr->clone());
    }
};

sim_info make_params(const ref_params* p) {
    sim_info s;
    s.Nx = p->nx;
    s.Ny = p->ny;
    s.x0 = p->x0;
    s.y0 = p->y0;
    s.dx = p->dx;
    s.dy = p->dy;
    s.numGC = (p->flux_solver == REF_FLUX_GODUNOV) ? 1 : 2;
    s.stclsize = s.numGC;
    s.BC_L = p->bc[0] ? "reflective" : "transmissive";
    s.BC_R = p->bc[1] ? "reflective" : "transmissive";
    s.BC_B = p->bc[2] ? "reflective" : "transmissive";
    s.BC_T = p->bc[3] ? "reflective" : "transmissive";
    s.T = p->T;
    s.CFL = p->cfl;
    s.output_freq = 0;
    s.outputname = "oracle";
    return s;
}

std::shared_ptr<OracleEuler> make_problem(const ref_params* p, const sim_info& s) {
    auto rs = std::make_shared<HLLC_riemann_solver_euler_equations>(s, p->gamma1, p->pinf1);
    std::shared_ptr<FluxSolverBaseEulerEquations> fs;
    if (p->flux_solver == REF_FLUX_GODUNOV)
        fs = std::make_shared<GodunovEulerEquations>(rs, s, p->gamma1, p->pinf1);
    else
        fs = std::make_shared<OracleMusclEuler>(rs, s, p->gamma1, p->pinf1, p->limiter,
                                                p->fix_dy_halfstep != 0);
    return std::make_shared<OracleEuler>(p->gamma1, p->pinf1, fs);
}

void to_grid(const double* a, int rows, int cols, gridtype& g) {
    g.assign(rows, rowtype(cols, vectype(4)));
    for (int i = 0; i < rows; ++i)
        for (int j = 0; j < cols; ++j)
            for (int k = 0; k < 4; ++k) g[i][j](k) = a[((size_t)i * cols + j) * 4 + k];
}

void from_grid(const gridtype& g, double* a) {
    int rows = (int)g.size(), cols = (int)g[0].size();
    for (int i = 0; i < rows; ++i)
        for (int j = 0; j < cols; ++j)
            for (int k = 0; k < 4; ++k) a[((size_t)i * cols + j) * 4 + k] = g[i][j](k);
}

}  // namespace

static double g_loop_seconds = 0.0;

extern "C" {

// Wall time of the time loop alone in the last *_run call (grid conversion
// excluded), for the CPU baseline.
double ref_euler_last_loop_seconds(void) { return g_loop_seconds; }

// Runs the reference time loop (headers/simulation.hpp:48-61):
//   while (t < T): dt = compute_dt(grid, n, t); advance_timestep(dt); t += dt;
//   n++; snap t to T within 1e-12
// stopping additionally after `max_steps` steps of this call.  `grid` is the
// reference's ghosted AoS grid ((ny+2g) x (nx+2g) x 4, row-major, rows = y)
// and is updated in place (ghost strips as the reference leaves them).
// `future` (same shape, may be null) holds the second buffer: the reference
// keeps two grids and swaps them, so stale ghost strips live in both.
// dt_log (may be null) receives each step's dt.  threads<=0 keeps OpenMP's
// default; 1 gives the deterministic order.
int ref_euler_run(const ref_params* p, double* grid, double* future, int max_steps, int* n_io,
                  double* t_io, double* dt_log, int threads) {
    if (threads > 0) omp_set_num_threads(threads);
    sim_info s = make_params(p);
    int g = s.numGC;
    int rows = p->ny + 2 * g, cols = p->nx + 2 * g;
    gridtype G, F;
    to_grid(grid, rows, cols, G);
    to_grid(future ? future : grid, rows, cols, F);
    auto prob = make_problem(p, s);
    std::shared_ptr<splitting_scheme_base> split;
    if (p->splitting == REF_SPLIT_STRANG) split = std::make_shared<strang_splitting>();
    else split = std::make_shared<naive_splitting>();
    int n = *n_io;
    double t = *t_io;
    int taken = 0;
    std::streambuf* old = std::cout.rdbuf();
    std::ostringstream sink;
    std::cout.rdbuf(sink.rdbuf());  // the reference prints on unphysical states
    double w0 = omp_get_wtime();
    while (t < s.T && taken < max_steps) {
        double dt = prob->compute_dt(G, s, n, t);
        split->advance_timestep(prob, G, F, s, dt, t);
        if (dt_log) dt_log[taken] = dt;
        t += dt;
        n++;
        taken++;
        if (std::fabs(t - s.T) < 1e-12) t = s.T;
    }
    g_loop_seconds = omp_get_wtime() - w0;
    std::cout.rdbuf(old);
    from_grid(G, grid);
    if (future) from_grid(F, future);
    *n_io = n;
    *t_io = t;
    return taken;
}

// Reference compute_dt (sourcecode/euler_timestep.cpp:7-44) on a ghosted grid.
double ref_euler_compute_dt(const ref_params* p, const double* grid, int n, double t) {
    sim_info s = make_params(p);
    int rows = p->ny + 2 * s.numGC, cols = p->nx + 2 * s.numGC;
    gridtype G;
    to_grid(grid, rows, cols, G);
    auto prob = make_problem(p, s);
    return prob->compute_dt(G, s, n, t);
}

// Reference flux for one face (flux_solver_MUSCLhancock.hpp:128-227 or the
// Godunov solver) from a stencil of 4 (or 2) conserved states.
void ref_euler_face_flux(const ref_params* p, const double* stencil, double dt, double dx,
                         double* flux, double* u_star) {
    sim_info s = make_params(p);
    auto prob = make_problem(p, s);
    int m = (p->flux_solver == REF_FLUX_GODUNOV) ? 2 : 4;
    std::vector<vectype> st(m, vectype(4));
    for (int c = 0; c < m; ++c)
        for (int k = 0; k < 4; ++k) st[c](k) = stencil[c * 4 + k];
    vectype f(4);
    double us = 0.0;
    std::streambuf* old = std::cout.rdbuf();
    std::ostringstream sink;
    std::cout.rdbuf(sink.rdbuf());
    prob->fs_ptr->flux_computation(st, f, dt, dx, us);
    std::cout.rdbuf(old);
    for (int k = 0; k < 4; ++k) flux[k] = f(k);
    *u_star = us;
}

// Reference set_ICs (sourcecode/euler_io.cpp:436-731) for one of its named
// test cases.  Writes the ghosted AoS grid and the parameters set_parameters
// chose (x0, y0, dx, dy, T, gamma, pinf, bc[4]).
int ref_euler_case_ic(const char* test_case, int nx, int ny, const char* flux_solver,
                      double* grid, ref_params* p_out) {
    settings_file SF;
    SF.Nx = nx;
    SF.Ny = ny;
    SF.CFL = 0.5;
    SF.splitting_scheme = "naive_splitting";
    SF.test_case = test_case;
    SF.output_freq = 0;
    SF.outputpath = "";
    SF.flux_solver = flux_solver;
    SF.riemann_solver = "HLLC";
    SF.problem = "euler";
    SF.basename = "oracle";
    Euler e;
    sim_info s;
    std::shared_ptr<gridtype> G = e.set_ICs(SF, s);
    from_grid(*G, grid);
    if (p_out) {
        p_out->nx = s.Nx;
        p_out->ny = s.Ny;
        p_out->x0 = s.x0;
        p_out->y0 = s.y0;
        p_out->dx = s.dx;
        p_out->dy = s.dy;
        p_out->T = s.T;
        p_out->gamma1 = e.eosparams.gamma;
        p_out->pinf1 = e.eosparams.pinf;
        p_out->bc[0] = s.BC_L == "reflective";
        p_out->bc[1] = s.BC_R == "reflective";
        p_out->bc[2] = s.BC_B == "reflective";
        p_out->bc[3] = s.BC_T == "reflective";
        p_out->flux_solver = s.numGC == 1 ? REF_FLUX_GODUNOV : REF_FLUX_MUSCL;
    }
    return 0;
}

// Reference IC helpers (sourcecode/euler_io.cpp:282-433) applied to a
// caller-supplied ghosted grid: kind 0 = add_circle_to_IC, 1 =
// add_rectangle_to_IC, 2 = set_circular_IC (W_out given in w_out).
int ref_euler_ic_shape(const ref_params* p, double* grid, int kind, const double* w_in,
                       const double* w_out, const double* geom, int nsamp) {
    sim_info s = make_params(p);
    int rows = p->ny + 2 * s.numGC, cols = p->nx + 2 * s.numGC;
    gridtype G;
    to_grid(grid, rows, cols, G);
    Euler e(p->gamma1, p->pinf1, nullptr);
    vectype Win(4), Wout(4);
    for (int k = 0; k < 4; ++k) {
        Win(k) = w_in[k];
        Wout(k) = w_out ? w_out[k] : 0.0;
    }
    if (kind == 0) e.add_circle_to_IC(Win, Eigen::Vector2d(geom[0], geom[1]), geom[2], G, s, nsamp);
    else if (kind == 1)
        e.add_rectangle_to_IC(Win, Eigen::Vector2d(geom[0], geom[1]), geom[2], geom[3], G, s, nsamp);
    else e.set_circular_IC(Win, Wout, Eigen::Vector2d(geom[0], geom[1]), geom[2], G, s, nsamp);
    from_grid(G, grid);
    return 0;
}

// Reference gnuplot writers (sourcecode/euler_io.cpp:1142-1216) for one grid.
int ref_euler_write(const ref_params* p, const double* grid, const char* basename, int n,
                    double t) {
    sim_info s = make_params(p);
    s.outputname = basename;
    int rows = p->ny + 2 * s.numGC, cols = p->nx + 2 * s.numGC;
    gridtype G;
    to_grid(grid, rows, cols, G);
    Euler e(p->gamma1, p->pinf1, nullptr);
    std::streambuf* old = std::cout.rdbuf();
    std::ostringstream sink;
    std::cout.rdbuf(sink.rdbuf());
    e.gnuplot_output(G, s, n, t);
    e.gnuplot_schlieren(G, s, n, t);
    std::cout.rdbuf(old);
    return 0;
}

// HOOK: the reference's main() (sourcecode/main.cpp:17-49):
// reads a settings file and runs simulation::run_simulation, which writes
// every output file with the reference's own cadence and writers.  Output
// state is static inside the reference (last output time), so run it once
// per process.
int ref_euler_simulate(const char* settings_path) {
    settings_file sf;
    sf.read_settings_file(settings_path);
    std::shared_ptr<problem_base> problem = std::make_shared<Euler>();
    simulation sim(sf, problem);
    return sim.run_simulation();
}

}  // extern "C"
