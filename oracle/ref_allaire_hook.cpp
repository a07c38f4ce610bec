// Oracle driver for the reference's Allaire five-equation solver.
//
// TEST INFRASTRUCTURE ONLY.  Compiled with the reference's allaire_2d sources
// (sourcecode/allaire_diffuse_{io,ppsweep,rowsweep,colsweep,timestep}.cpp and
// headers/) into oracle/_ref/libref_allaire.so by oracle/Makefile.  The
// reference's own main() is not linked: as shipped it instantiates Euler,
// whose sources are absent from allaire_2d (sourcecode/main.cpp:27-36), so
// the unmodified tree does not link.
//
// Hooks (each labelled HOOK below):
//   * selectable slope limiter that survives clone() (the reference hard-wires
//     minmod, headers/flux_solver_MUSCLhancock.hpp:268) plus van Leer;
//   * HLLC with PVRS-based wave speeds, restated from the commented-out block
//     at headers/riemann_solver_HLLC.hpp:84-107 with p* from the PVRS solver
//     (headers/riemann_solver_PVRS.hpp:85) and the shock-speed jump of
//     headers/mixturemodel.hpp:42-52; everything after the speeds follows
//     headers/riemann_solver_HLLC.hpp:111-149;
//   * volume-fraction clip [z_min, 1-z_min] in the second-order z update
//     (the reference clips to [0,1], headers/zupdate.hpp:62-67);
//   * optional dy in the y-sweep half-step (the reference passes params.dx,
//     sourcecode/allaire_diffuse_colsweep.cpp:42).
#include <algorithm>
#include <cassert>
#include <cmath>
#include <cstring>
#include <fstream>
#include <functional>
#include <iostream>
#include <memory>
#include <sstream>
#include <string>
#include <vector>
#include <omp.h>
#include <Eigen/Dense>

#define private public
#define protected public
#include "allaire_diffuse.hpp"
#include "flux_solver_MUSCLhancock.hpp"
#include "flux_solver_godunov.hpp"
#include "riemann_solver_HLLC.hpp"
#include "mixturemodel.hpp"
#include "misc.hpp"
#include "zupdate.hpp"
#include "splitting_scheme.hpp"
#include "settings_file.hpp"
#include "simulation.hpp"
#undef private
#undef protected

#include "ref_common.h"

namespace {

vectype vanleer_slope(const vectype& dL, const vectype& dR) {
    vectype s(dL.rows());
    for (int k = 0; k < dL.rows(); ++k) {
        if (dL(k) * dR(k) > 0.0) s(k) = (2.0 * dL(k) * dR(k)) / (dL(k) + dR(k));
        else s(k) = 0.0;
    }
    return s;
}

std::function<vectype(const vectype&, const vectype&)> pick_limiter(int lim) {
    switch (lim) {
        case REF_LIM_MINMOD: return minmod_limited_slope;
        case REF_LIM_VANLEER: return vanleer_slope;
        case REF_LIM_MC: return MC_limited_slope;
        case REF_LIM_UNLIMITED: return unlimited_central_diff;
    }
    return minmod_limited_slope;
}

// HOOK: HLLC with PVRS wave-speed estimates for the mixture model.
class OracleHLLCPVRS : public riemann_solver_base {
public:
    OracleHLLCPVRS(sim_info p, double g1, double g2, double p1, double p2)
        : riemann_solver_base(p, g1, g2, p1, p2) {}

    vectype solve_RP(const vectype& UL, const vectype& UR, double* u_star_ptr = nullptr,
                     double* p_star_ptr = nullptr, double* v_star_ptr = nullptr) override {
        const binarySGparams& eo = eosparams;
        double zl = UL(5), rl = UL(0) + UL(1);
        double ul = UL(2) / rl, vl = UL(3) / rl;
        double el = UL(4) / rl - 0.5 * (ul * ul + vl * vl);
        double pl = allairemodel::mixture_pressure(eo, rl, el, zl);
        double cl = allairemodel::mixture_soundspeed(eo, rl, pl, zl);
        double zr = UR(5), rr = UR(0) + UR(1);
        double ur = UR(2) / rr, vr = UR(3) / rr;
        double er = UR(4) / rr - 0.5 * (ur * ur + vr * vr);
        double pr = allairemodel::mixture_pressure(eo, rr, er, zr);
        double cr = allairemodel::mixture_soundspeed(eo, rr, pr, zr);

        // Wave speeds: PVRS star pressure, exact shock speed on a compressive side.
        double rho_avg = 0.5 * (rl + rr);
        double c_avg = 0.5 * (cl + cr);
        double ppv = std::max(0.0, 0.5 * (pl + pr) + 0.5 * (ul - ur) * rho_avg * c_avg);
        double sl = (ppv > pl) ? ul - allairemodel::shock_speed_jump(eo, pl, rl, ppv, zl) : ul - cl;
        double sr = (ppv > pr) ? ur + allairemodel::shock_speed_jump(eo, pr, rr, ppv, zr) : ur + cr;

        double us = (pr - pl + rl * ul * (sl - ul) - rr * ur * (sr - ur)) /
                    (rl * (sl - ul) - rr * (sr - ur));
        double ps = pl + rl * (sl - ul) * (us - ul);
        double fl = (sl - ul) / (sl - us);
        double fr = (sr - ur) / (sr - us);
        if (u_star_ptr) *u_star_ptr = us;
        if (p_star_ptr) *p_star_ptr = ps;
        if (v_star_ptr) *v_star_ptr = (us >= 0.0) ? vl : vr;

        vectype sL(6), sR(6);
        sL(0) = fl * UL(0);
        sL(1) = fl * UL(1);
        sL(2) = fl * rl * us;
        sL(3) = fl * UL(3);
        sL(4) = fl * (UL(4) + (us - ul) * (rl * us + (pl / (sl - ul))));
        sL(5) = 0.0;
        sR(0) = fr * UR(0);
        sR(1) = fr * UR(1);
        sR(2) = fr * rr * us;
        sR(3) = fr * UR(3);
        sR(4) = fr * (UR(4) + (us - ur) * (rr * us + (pr / (sr - ur))));
        sR(5) = 0.0;
        double cs = std::copysign(1.0, us);
        vectype f = ((1.0 + cs) / 2.0) * (flux_conserved_var(eo, UL) + std::min(0.0, sl) * (sL - UL)) +
                    ((1.0 - cs) / 2.0) * (flux_conserved_var(eo, UR) + std::max(0.0, sr) * (sR - UR));
        f(5) = 0.0;
        return f;
    }
    std::shared_ptr<riemann_solver_base> clone() override {
        return std::make_shared<OracleHLLCPVRS>(params, eosparams.gamma1, eosparams.gamma2,
                                                eosparams.pinf1, eosparams.pinf2);
    }
};

// HOOK: second-order z update with the clip interval [zmin, 1-zmin].
class OracleZClip : public zupdate_base {
public:
    double zmin;
    explicit OracleZClip(double zmin_) : zmin(zmin_) {}
    double zupdate(double dx, double dt, double zL, double z, double zR, double usL, double usR,
                   double zsL, double zsR) override {
        double nz = z - (dt / dx) * (usR * zsR - usL * zsL - z * (usR - usL));
        return std::max(std::min(1.0 - zmin, nz), zmin);
    }
    std::shared_ptr<zupdate_base> clone() override { return std::make_shared<OracleZClip>(zmin); }
};

// HOOK: limiter selection that survives clone(), optional dy half-step.
class OracleMusclAllaire : public flux_solver_MUSCLHANCOCK {
public:
    int lim;
    bool fix_dy;
    bool in_col = false;
    OracleMusclAllaire(std::shared_ptr<riemann_solver_base> rs, sim_info p, double g1, double g2,
                       double p1, double p2, int lim_, bool fix_dy_)
        : flux_solver_MUSCLHANCOCK(rs, p, g1, g2, p1, p2), lim(lim_), fix_dy(fix_dy_) {
        slopelimiter = pick_limiter(lim);
    }
    void flux_computation(const std::vector<vectype>& stencil, vectype& flux, double dt, double dx,
                          double& u_star, double& z_star, double* p_star_ptr = nullptr,
                          double* v_star_ptr = nullptr) override {
        double h = (in_col && fix_dy) ? params.dy : dx;
        flux_solver_MUSCLHANCOCK::flux_computation(stencil, flux, dt, h, u_star, z_star, p_star_ptr,
                                                   v_star_ptr);
    }
    std::shared_ptr<flux_solver_base> clone() override {
        return std::make_shared<OracleMusclAllaire>(RS_ptr->clone(), params, eosparams.gamma1,
                                                    eosparams.gamma2, eosparams.pinf1,
                                                    eosparams.pinf2, lim, fix_dy);
    }
};

class OracleAllaire : public allaire_diffuse {
public:
    OracleAllaire(double g1, double g2, double p1, double p2, std::shared_ptr<flux_solver_base> fs,
                  std::shared_ptr<zupdate_base> zu)
        : allaire_diffuse(g1, g2, p1, p2, fs, zu) {}
    void update_col(const gridtype& grid, gridtype& future_grid, const sim_info& params, int j,
                    double dt, double t) override {
        OracleMusclAllaire* m = dynamic_cast<OracleMusclAllaire*>(FS_ptr.get());
        if (m) m->in_col = true;
        allaire_diffuse::update_col(grid, future_grid, params, j, dt, t);
        if (m) m->in_col = false;
    }
    std::shared_ptr<problem_base> clone() override {
        return std::make_shared<OracleAllaire>(eosparams.gamma1, eosparams.gamma2, eosparams.pinf1,
                                               eosparams.pinf2, FS_ptr->clone(),
                                               zupdate_ptr->clone());
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

std::shared_ptr<OracleAllaire> make_problem(const ref_params* p, const sim_info& s) {
    std::shared_ptr<riemann_solver_base> rs;
    if (p->wavespeed == REF_WS_PVRS)
        rs = std::make_shared<OracleHLLCPVRS>(s, p->gamma1, p->gamma2, p->pinf1, p->pinf2);
    else
        rs = std::make_shared<HLLC_riemann_solver>(s, p->gamma1, p->gamma2, p->pinf1, p->pinf2);
    std::shared_ptr<flux_solver_base> fs;
    std::shared_ptr<zupdate_base> zu;
    if (p->flux_solver == REF_FLUX_GODUNOV) {
        fs = std::make_shared<flux_solver_godunov>(rs, s, p->gamma1, p->gamma2, p->pinf1, p->pinf2);
        zu = std::make_shared<zupdate_upwind>();
    } else {
        fs = std::make_shared<OracleMusclAllaire>(rs, s, p->gamma1, p->gamma2, p->pinf1, p->pinf2,
                                                  p->limiter, p->fix_dy_halfstep != 0);
        if (p->z_min > 0.0) zu = std::make_shared<OracleZClip>(p->z_min);
        else zu = std::make_shared<zupdate_secondorder>();
    }
    return std::make_shared<OracleAllaire>(p->gamma1, p->gamma2, p->pinf1, p->pinf2, fs, zu);
}

void to_grid(const double* a, int rows, int cols, gridtype& g) {
    g.assign(rows, rowtype(cols, vectype(6)));
    for (int i = 0; i < rows; ++i)
        for (int j = 0; j < cols; ++j)
            for (int k = 0; k < 6; ++k) g[i][j](k) = a[((size_t)i * cols + j) * 6 + k];
}

void from_grid(const gridtype& g, double* a) {
    int rows = (int)g.size(), cols = (int)g[0].size();
    for (int i = 0; i < rows; ++i)
        for (int j = 0; j < cols; ++j)
            for (int k = 0; k < 6; ++k) a[((size_t)i * cols + j) * 6 + k] = g[i][j](k);
}

// Assertion guard: the reference aborts through assert() on an unphysical
// state.  The oracle keeps asserts live but reports them instead of aborting
// the test process by checking the same predicate first.
}  // namespace

static double g_loop_seconds = 0.0;

extern "C" {

// Wall time of the time loop alone in the last *_run call (grid conversion
// excluded), for the CPU baseline.
double ref_allaire_last_loop_seconds(void) { return g_loop_seconds; }

// Same contract as ref_euler_run (oracle/ref_euler_hook.cpp) for the Allaire
// model: ghosted AoS grid with 6 stored components per cell.
int ref_allaire_run(const ref_params* p, double* grid, double* future, int max_steps, int* n_io,
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
    std::cout.rdbuf(sink.rdbuf());
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

double ref_allaire_compute_dt(const ref_params* p, const double* grid, int n, double t) {
    sim_info s = make_params(p);
    int rows = p->ny + 2 * s.numGC, cols = p->nx + 2 * s.numGC;
    gridtype G;
    to_grid(grid, rows, cols, G);
    auto prob = make_problem(p, s);
    return prob->compute_dt(G, s, n, t);
}

// One face of the reference MUSCL-Hancock + HLLC solver
// (flux_solver_MUSCLhancock.hpp:272-376): flux(6), u*, z*.
void ref_allaire_face_flux(const ref_params* p, const double* stencil, double dt, double dx,
                           double* flux, double* u_star, double* z_star) {
    sim_info s = make_params(p);
    auto prob = make_problem(p, s);
    int m = (p->flux_solver == REF_FLUX_GODUNOV) ? 2 : 4;
    std::vector<vectype> st(m, vectype(6));
    for (int c = 0; c < m; ++c)
        for (int k = 0; k < 6; ++k) st[c](k) = stencil[c * 6 + k];
    vectype f(6);
    double us = 0.0, zs = 0.0;
    std::streambuf* old = std::cout.rdbuf();
    std::ostringstream sink;
    std::cout.rdbuf(sink.rdbuf());
    prob->FS_ptr->flux_computation(st, f, dt, dx, us, zs);
    std::cout.rdbuf(old);
    for (int k = 0; k < 6; ++k) flux[k] = f(k);
    *u_star = us;
    *z_star = zs;
}

// Reference set_ICs (sourcecode/allaire_diffuse_io.cpp:312-990) for a named case.
int ref_allaire_case_ic(const char* test_case, int nx, int ny, const char* flux_solver,
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
    SF.problem = "allaire";
    SF.basename = "oracle";
    allaire_diffuse a;
    sim_info s;
    std::shared_ptr<gridtype> G = a.set_ICs(SF, s);
    from_grid(*G, grid);
    if (p_out) {
        p_out->nx = s.Nx;
        p_out->ny = s.Ny;
        p_out->x0 = s.x0;
        p_out->y0 = s.y0;
        p_out->dx = s.dx;
        p_out->dy = s.dy;
        p_out->T = s.T;
        p_out->gamma1 = a.eosparams.gamma1;
        p_out->gamma2 = a.eosparams.gamma2;
        p_out->pinf1 = a.eosparams.pinf1;
        p_out->pinf2 = a.eosparams.pinf2;
        p_out->bc[0] = s.BC_L == "reflective";
        p_out->bc[1] = s.BC_R == "reflective";
        p_out->bc[2] = s.BC_B == "reflective";
        p_out->bc[3] = s.BC_T == "reflective";
        p_out->flux_solver = s.numGC == 1 ? REF_FLUX_GODUNOV : REF_FLUX_MUSCL;
    }
    return 0;
}

// Reference gnuplot writers (sourcecode/allaire_diffuse_io.cpp:1109-1232).
int ref_allaire_write(const ref_params* p, const double* grid, const char* basename, int n,
                      double t) {
    sim_info s = make_params(p);
    s.outputname = basename;
    int rows = p->ny + 2 * s.numGC, cols = p->nx + 2 * s.numGC;
    gridtype G;
    to_grid(grid, rows, cols, G);
    allaire_diffuse a(p->gamma1, p->gamma2, p->pinf1, p->pinf2, nullptr, nullptr);
    std::streambuf* old = std::cout.rdbuf();
    std::ostringstream sink;
    std::cout.rdbuf(sink.rdbuf());
    a.gnuplot_output(G, s, n, t);
    a.gnuplot_schlieren(G, s, n, t);
    a.gnuplot_lineout(G, s, n, t);
    std::cout.rdbuf(old);
    return 0;
}

// HOOK: the reference's main() (sourcecode/main.cpp:17-49, with the allaire_diffuse problem its commented line 36 names):
// reads a settings file and runs simulation::run_simulation, which writes
// every output file with the reference's own cadence and writers.  Output
// state is static inside the reference (last output time), so run it once
// per process.
int ref_allaire_simulate(const char* settings_path) {
    settings_file sf;
    sf.read_settings_file(settings_path);
    std::shared_ptr<problem_base> problem = std::make_shared<allaire_diffuse>();
    simulation sim(sf, problem);
    return sim.run_simulation();
}

}  // extern "C"
