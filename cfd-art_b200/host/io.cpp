// settingsfile.txt parsing and the reference's gnuplot output formats.
#include <algorithm>
#include <cmath>
#include <cstring>
#include <fstream>
#include <sstream>
#include <string>
#include <vector>

#include "../../include/cfdgpu.h"
#include "../../include/cfdgpu_host.h"
#include "cfd_checkpoint.h"
#include "cfd_error.h"

namespace {

void copy_str(char* dst, size_t n, const std::string& s) {
    strncpy(dst, s.c_str(), n - 1);
    dst[n - 1] = 0;
}

struct View {
    int nx, ny, g, nv;
    double x0, y0, dx, dy;
    const double* a;
    const double* cell(int i, int j) const { return a + ((size_t)i * (nx + 2 * g) + j) * nv; }
    double ccx(int j) const { return x0 + double(j - g) * dx + 0.5 * dx; }
    double ccy(int i) const { return y0 + double(i - g) * dy + 0.5 * dy; }
};

View view_of(const cfd_config* c, const double* grid) {
    View v;
    v.nx = c->nx;
    v.ny = c->ny;
    v.g = c->flux_solver == CFD_FLUX_GODUNOV ? 1 : 2;
    v.nv = cfd_nvar(c->model);
    v.x0 = c->x0;
    v.y0 = c->y0;
    v.dx = c->dx;
    v.dy = c->dy;
    v.a = grid;
    return v;
}

double density(const cfd_config* c, const double* U) {
    return c->model == CFD_MODEL_EULER ? U[0] : U[0] + U[1];
}

// A/headers/mixturemodel.hpp:18-24
double mixture_pressure(const cfd_config* c, double rho, double e, double z) {
    double eps = z / (c->gamma1 - 1.0) + (1.0 - z) / (c->gamma2 - 1.0);
    double k = (z * c->gamma1 * c->pinf1 / (c->gamma1 - 1.0) +
                (1.0 - z) * c->gamma2 * c->pinf2 / (c->gamma2 - 1.0)) /
               eps;
    return rho * e / eps - k;
}

// Values of the optional settings keys; -1 for a value the key does not take.
int lim_of(const std::string& s) {
    if (s == "minmod") return CFD_LIM_MINMOD;
    if (s == "vanleer" || s == "van_leer") return CFD_LIM_VANLEER;
    if (s == "mc" || s == "MC") return CFD_LIM_MC;
    if (s == "unlimited") return CFD_LIM_UNLIMITED;
    return -1;
}

int wavespeed_of(const std::string& s) {
    if (s == "davis") return CFD_WS_DAVIS;
    if (s == "pvrs") return CFD_WS_PVRS;
    return -1;
}

int precision_of(const std::string& s) {
    if (s == "fp64") return CFD_PREC_FP64;
    if (s == "mixed") return CFD_PREC_MIXED;
    if (s == "fp64_fast") return CFD_PREC_FP64_FAST;
    return -1;
}

int cannot_write(const std::string& name) {
    return cfd_fail(CFD_ERR_INVALID, "cannot open output file '%s'", name.c_str());
}

int recipe_of(const std::string& tc) {
    if (tc == "four_quadrant") return CFD_RECIPE_FOUR_QUADRANT;
    if (tc == "shock_bubbles") return CFD_RECIPE_SHOCK_BUBBLES;
    if (tc == "water_shock_air_bubble") return CFD_RECIPE_WATER_SHOCK_AIR_BUBBLE;
    return 0;
}

}  // namespace

extern "C" {

// headers/settings_file.hpp:35-71
int cfd_read_settings(const char* path, cfd_settings* s) {
    if (!path || !s) return cfd_fail(CFD_ERR_INVALID, "cfd_read_settings: null argument");
    memset(s, 0, sizeof *s);
    s->seed = 20261203ULL;
    s->nbubbles = 32;
    std::ifstream in(path);
    if (!in) return cfd_fail(CFD_ERR_INVALID, "cannot open settings file '%s'", path);
    std::string line;
    while (std::getline(in, line)) {
        std::istringstream iss(line);
        std::string key, val;
        iss >> key;
        if (key == "Nx") iss >> s->Nx;
        else if (key == "Ny") iss >> s->Ny;
        else if (key == "CFL") iss >> s->CFL;
        else if (key == "output_freq") iss >> s->output_freq;
        else if (key == "steps") iss >> s->steps;
        else if (key == "alpha_clip") iss >> s->alpha_clip;
        else if (key == "fix_dy_halfstep") iss >> s->fix_dy_halfstep;
        else if (key == "seed") iss >> s->seed;
        else if (key == "nbubbles") iss >> s->nbubbles;
        else {
            iss >> val;
            if (key == "splitting_scheme") copy_str(s->splitting_scheme, sizeof s->splitting_scheme, val);
            else if (key == "test_case") copy_str(s->test_case, sizeof s->test_case, val);
            else if (key == "outputpath") copy_str(s->outputpath, sizeof s->outputpath, val);
            else if (key == "flux_solver") copy_str(s->flux_solver, sizeof s->flux_solver, val);
            else if (key == "riemann_solver") copy_str(s->riemann_solver, sizeof s->riemann_solver, val);
            else if (key == "problem") copy_str(s->problem, sizeof s->problem, val);
            else if (key == "precision") copy_str(s->precision, sizeof s->precision, val);
            else if (key == "limiter") copy_str(s->limiter, sizeof s->limiter, val);
            else if (key == "wavespeed") copy_str(s->wavespeed, sizeof s->wavespeed, val);
        }
    }
    std::string base = std::string(s->outputpath) + s->problem + "-" + s->test_case + "-" +
                       s->flux_solver + "-" + std::to_string(s->Nx) + "-" + std::to_string(s->Ny);
    copy_str(s->basename, sizeof s->basename, base);
    return CFD_OK;
}

int cfd_settings_config(const cfd_settings* s, cfd_config* cfg) {
    if (!s || !cfg) return cfd_fail(CFD_ERR_INVALID, "cfd_settings_config: null argument");
    std::string prob = s->problem;
    int model = (prob == "allaire" || prob == "allaire_diffuse") ? CFD_MODEL_ALLAIRE
                                                                 : CFD_MODEL_EULER;
    if (prob != "euler" && model == CFD_MODEL_EULER)
        return cfd_fail(CFD_ERR_INVALID, "settings: unknown problem '%s' (euler, allaire)",
                        s->problem);
    std::string fs = s->flux_solver;
    int flux;
    if (fs == "MUSCL") flux = CFD_FLUX_MUSCL;
    else if (fs == "Godunov") flux = CFD_FLUX_GODUNOV;
    else
        return cfd_fail(CFD_ERR_INVALID, "settings: unknown flux_solver '%s' (MUSCL, Godunov)",
                        s->flux_solver);
    if (std::string(s->riemann_solver) != "HLLC")
        return cfd_fail(CFD_ERR_INVALID, "settings: unknown riemann_solver '%s' (HLLC)",
                        s->riemann_solver);
    std::string sp = s->splitting_scheme;
    int split;
    if (sp == "naive_splitting") split = CFD_SPLIT_NAIVE;
    else if (sp == "strang_splitting") split = CFD_SPLIT_STRANG;
    else
        return cfd_fail(CFD_ERR_INVALID,
                        "settings: unknown splitting_scheme '%s' (naive_splitting, "
                        "strang_splitting)",
                        s->splitting_scheme);
    int lim = s->limiter[0] ? lim_of(s->limiter) : 0;
    if (lim < 0)
        return cfd_fail(CFD_ERR_INVALID,
                        "settings: unknown limiter '%s' (minmod, vanleer, mc, unlimited)",
                        s->limiter);
    int ws = s->wavespeed[0] ? wavespeed_of(s->wavespeed) : 0;
    if (ws < 0)
        return cfd_fail(CFD_ERR_INVALID, "settings: unknown wavespeed '%s' (davis, pvrs)",
                        s->wavespeed);
    int prec = s->precision[0] ? precision_of(s->precision) : CFD_PREC_FP64;
    if (prec < 0)
        return cfd_fail(CFD_ERR_INVALID, "settings: unknown precision '%s' (fp64, mixed, fp64_fast)",
                        s->precision);
    int r;
    int rec = recipe_of(s->test_case);
    if (rec) r = cfd_recipe_config(rec, s->Nx, s->Ny, cfg);
    else r = cfd_case_config(model, s->test_case, s->Nx, s->Ny, flux, cfg);
    if (r) return r;  // with its message
    if (rec && cfg->model != model)
        return cfd_fail(CFD_ERR_INVALID, "settings: test_case '%s' is not a %s problem",
                        s->test_case, s->problem);
    cfg->flux_solver = flux;
    cfg->cfl = s->CFL;
    cfg->splitting = split;
    if (s->limiter[0]) cfg->limiter = lim;
    if (s->wavespeed[0]) cfg->wavespeed = ws;
    if (s->alpha_clip > 0.0) cfg->z_min = s->alpha_clip;
    cfg->fix_dy_halfstep = s->fix_dy_halfstep;
    cfg->precision = prec;
    return CFD_OK;
}

int cfd_settings_ic(const cfd_settings* s, const cfd_config* cfg, double* grid) {
    int rec = recipe_of(s->test_case);
    if (rec) return cfd_recipe_ic(cfg, rec, s->seed, s->nbubbles, grid);
    return cfd_case_ic(cfg, s->test_case, s->seed, grid);
}

// E/sourcecode/euler_io.cpp:1188-1216, A/sourcecode/allaire_diffuse_io.cpp:1155-1186
int cfd_write_state(const cfd_config* c, const double* grid, const char* basename, double t) {
    if (!c || !grid || !basename) return cfd_fail(CFD_ERR_INVALID, "cfd_write_state: null argument");
    View v = view_of(c, grid);
    const std::string name = std::string(basename) + "-state-" + std::to_string(t) + ".dat";
    std::ofstream out(name);
    if (!out) return cannot_write(name);
    for (int i = v.g; i < v.ny + v.g; ++i) {
        for (int j = v.g; j < v.nx + v.g; ++j) {
            const double* U = v.cell(i, j);
            double x = v.ccx(j), y = v.ccy(i);
            if (c->model == CFD_MODEL_EULER) {
                double rho = U[0];
                double u = U[1] / rho;
                double vv = U[2] / rho;
                double E = U[3];
                double e = E / rho - 0.5 * (u * u + vv * vv);
                // the reference passes (rho, e) in swapped order to eos::pressure
                double p = (c->gamma1 - 1.0) * e * rho - c->gamma1 * c->pinf1;
                out << x << " " << y << " " << rho << " " << u << " " << vv << " " << e << " " << p
                    << std::endl;
            } else {
                double rho = U[0] + U[1];
                double u = U[2] / rho;
                double vv = U[3] / rho;
                double E = U[4];
                double e = E / rho - 0.5 * (u * u + vv * vv);
                double z = U[5];
                double p = mixture_pressure(c, rho, e, z);
                out << x << " " << y << " " << rho << " " << u << " " << vv << " " << e << " " << z
                    << " " << p << std::endl;
            }
        }
        out << std::endl;
    }
    return CFD_OK;
}

// E/sourcecode/euler_io.cpp:1142-1185 (A: :1109-1150): |grad rho| / max.
int cfd_write_schlieren(const cfd_config* c, const double* grid, const char* basename, double t) {
    if (!c || !grid || !basename)
        return cfd_fail(CFD_ERR_INVALID, "cfd_write_schlieren: null argument");
    View v = view_of(c, grid);
    std::vector<double> g;
    g.reserve((size_t)v.nx * v.ny);
    for (int i = v.g; i < v.ny + v.g; ++i)
        for (int j = v.g; j < v.nx + v.g; ++j) {
            double rl = density(c, v.cell(i, j - 1)), rr = density(c, v.cell(i, j + 1));
            double rt = density(c, v.cell(i + 1, j)), rb = density(c, v.cell(i - 1, j));
            double gx = (rr - rl) / (2.0 * v.dx);
            double gy = (rt - rb) / (2.0 * v.dy);
            g.push_back(std::sqrt(gx * gx + gy * gy));
        }
    return cfd_write_schlieren_field(c, g.data(), basename, t);
}

int cfd_write_schlieren_field(const cfd_config* c, const double* field, const char* basename,
                              double t) {
    if (!c || !field || !basename)
        return cfd_fail(CFD_ERR_INVALID, "cfd_write_schlieren_field: null argument");
    const size_t n = (size_t)c->nx * c->ny;
    double mx = *std::max_element(field, field + n);
    const std::string name = std::string(basename) + "-schlieren-" + std::to_string(t) + ".dat";
    std::ofstream out(name);
    if (!out) return cannot_write(name);
    size_t k = 0;
    for (int i = 0; i < c->ny; ++i) {
        const double y = c->y0 + double(i) * c->dy + 0.5 * c->dy;  // cell centres as View
        for (int j = 0; j < c->nx; ++j) {
            const double x = c->x0 + double(j) * c->dx + 0.5 * c->dx;
            out << x << " " << y << " " << field[k] / mx << std::endl;
            ++k;
        }
        out << std::endl;
    }
    return CFD_OK;
}

// A/sourcecode/allaire_diffuse_io.cpp:1188-1232: row Ny/2 and column Nx/2
// of the ghosted grid (ghost cells included), -lineoutx-<n>.dat and
// -lineouty-<n>.dat.
int cfd_write_lineout(const cfd_config* c, const double* grid, const char* basename, int n) {
    if (!c || !grid || !basename) return cfd_fail(CFD_ERR_INVALID, "cfd_write_lineout: null argument");
    if (c->model != CFD_MODEL_ALLAIRE)
        return cfd_fail(CFD_ERR_INVALID, "cfd_write_lineout: Allaire grids only");
    View v = view_of(c, grid);
    auto line = [&](std::ofstream& out, double coord, const double* U) {
        double rho = U[0] + U[1];
        double u = U[2] / rho;
        double vv = U[3] / rho;
        double e = U[4] / rho - 0.5 * (u * u + vv * vv);
        double z = U[5];
        double p = mixture_pressure(c, rho, e, z);
        out << coord << " " << rho << " " << u << " " << vv << " " << e << " " << p << " " << z
            << std::endl;
    };
    const std::string xname = std::string(basename) + "-lineoutx-" + std::to_string(n) + ".dat";
    std::ofstream ox(xname);
    if (!ox) return cannot_write(xname);
    int i = v.ny / 2;
    for (int j = 0; j < v.nx + 2 * v.g; ++j) line(ox, v.ccx(j), v.cell(i, j));
    ox.close();
    const std::string yname = std::string(basename) + "-lineouty-" + std::to_string(n) + ".dat";
    std::ofstream oy(yname);
    if (!oy) return cannot_write(yname);
    int j = v.nx / 2;
    for (int r = 0; r < v.ny + 2 * v.g; ++r) line(oy, v.ccy(r), v.cell(r, j));
    return CFD_OK;
}

int cfd_checkpoint_info(const char* path, cfd_config* cfg, int* n, double* t) {
    if (!path) return cfd_fail(CFD_ERR_INVALID, "cfd_checkpoint_info: null path");
    FILE* f = fopen(path, "rb");
    if (!f) return cfd_fail(CFD_ERR_INVALID, "cannot open checkpoint '%s'", path);
    cfd::CkptHeader h;
    int r = cfd::ckpt_read_header(f, h);
    fclose(f);
    if (r) return r;
    if (cfg) *cfg = h.cfg;
    if (n) *n = h.n;
    if (t) *t = h.t;
    return CFD_OK;
}

int cfd_write_masschange(const cfd_config* c, const char* basename, int nrec, const double* t,
                         const double* m1, const double* m2) {
    if (!c || !basename || nrec < 1 || !t || !m1)
        return cfd_fail(CFD_ERR_INVALID, "cfd_write_masschange: null argument or no records");
    if (c->model == CFD_MODEL_ALLAIRE && !m2)
        return cfd_fail(CFD_ERR_INVALID, "cfd_write_masschange: Allaire needs both mass series");
    const std::string name = std::string(basename) + "-masschange.dat";
    std::ofstream out(name);
    if (!out) return cannot_write(name);
    for (int k = 0; k < nrec; ++k) {
        if (c->model == CFD_MODEL_EULER)
            out << t[k] << " " << m1[k] - m1[0] << std::endl;
        else
            out << t[k] << " " << (m1[k] - m1[0]) / m1[0] << " " << (m2[k] - m2[0]) / m2[0]
                << std::endl;
    }
    return CFD_OK;
}

}  // extern "C"
