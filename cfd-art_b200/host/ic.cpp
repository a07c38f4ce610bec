// Initial-condition hooks, on the host, in the reference's ghosted AoS layout.
//
// Named test cases restate the reference's set_parameters / set_ICs
// (E/sourcecode/euler_io.cpp:13-234, 436-731 and
// A/sourcecode/allaire_diffuse_io.cpp:13-310, 401-990) with the same sample
// positions and arithmetic, so the grids are bit-identical to the
// reference's (checked by the tests).  The seeded workload recipes
// (four-quadrant Riemann problem, shock + bubbles, water shock on an air
// bubble) are new ICs built from the same helpers.
//
// Every recipe and every named case made of the reference's shape helpers is
// expressed as a shape program (csrc/ic_program.h) that the host evaluates
// here and the device evaluates in csrc/cfd_ic.cu; the four Allaire cases
// with their own per-cell formulas (shocked_SF6, TSTM, RMI_SF6,
// tin_air_implosion) are shape-program operations too (MIXED_CELL,
// RING_CELL).
#include <cmath>
#include <cstdint>
#include <cstring>
#include <random>
#include <string>
#include <vector>

#include "../../include/cfdgpu.h"
#include "../../include/cfdgpu_host.h"
#include "cfd_error.h"
#include "ic_builders.h"

using cfdic::Op;

namespace {

struct Grid {
    int nx, ny, g, nv;
    double x0, y0, dx, dy;
    double* a;
    double* cell(int i, int j) { return a + ((size_t)i * (nx + 2 * g) + j) * nv; }
    int rows() const { return ny + 2 * g; }
    int cols() const { return nx + 2 * g; }
    // headers/sim_info.hpp:40-46
    double ccx(int j) const { return x0 + double(j - g) * dx + 0.5 * dx; }
    double ccy(int i) const { return y0 + double(i - g) * dy + 0.5 * dy; }
};

Grid make_grid(const cfd_config* cfg, double* grid) {
    Grid G;
    G.nx = cfg->nx;
    G.ny = cfg->ny;
    G.g = cfg->flux_solver == CFD_FLUX_GODUNOV ? 1 : 2;
    G.nv = cfd_nvar(cfg->model);
    G.x0 = cfg->x0;
    G.y0 = cfg->y0;
    G.dx = cfg->dx;
    G.dy = cfg->dy;
    G.a = grid;
    return G;
}

cfdic::Eos make_eos(const cfd_config* cfg) {
    cfdic::Eos q;
    q.model = cfg->model == CFD_MODEL_EULER ? 0 : 1;
    q.g1 = cfg->gamma1;
    q.p1 = cfg->pinf1;
    q.g2 = cfg->gamma2;
    q.p2 = cfg->pinf2;
    return q;
}

// Runs a shape program over every cell of the ghosted grid.
void run_program(Grid& G, const std::vector<Op>& ops, const cfdic::Eos& q) {
    cfdic::Geom geo{G.x0, G.y0, G.dx, G.dy};
    for (int i = 0; i < G.rows(); ++i)
        for (int j = 0; j < G.cols(); ++j)
            cfdic::eval_cell(ops.data(), (int)ops.size(), q, geo, i - G.g, j - G.g, G.cell(i, j));
}

// --------------------------------------------------------- op emitters ---
struct Prog {
    const cfdic::Eos& q;
    std::vector<Op>& ops;
    int nv() const { return cfdic::nvar(q); }
    Op& push(int kind, int n = 10) {
        Op o;
        memset(&o, 0, sizeof o);
        o.kind = kind;
        o.n = n;
        ops.push_back(o);
        return ops.back();
    }
    void copy(double* dst, const double* src) const { memcpy(dst, src, sizeof(double) * nv()); }
    void fill(const double* U) { copy(push(cfdic::OP_FILL).v[0], U); }
    // E/sourcecode/euler_io.cpp:335-389
    void add_circle(const double* U, double cx, double cy, double R, int N = 10) {
        Op& o = push(cfdic::OP_ADD_CIRCLE, N);
        o.a[0] = cx, o.a[1] = cy, o.a[2] = R;
        copy(o.v[0], U);
    }
    // E/sourcecode/euler_io.cpp:282-330
    void add_rect(const double* U, double blx, double bly, double w, double h, int N = 10) {
        Op& o = push(cfdic::OP_ADD_RECT, N);
        o.a[0] = blx, o.a[1] = bly, o.a[2] = w, o.a[3] = h;
        copy(o.v[0], U);
    }
    // E/sourcecode/euler_io.cpp:392-433, A/sourcecode/allaire_diffuse_io.cpp:358-399
    void set_circular(const double* W_in, const double* W_out, double cx, double cy, double R,
                      int N) {
        Op& o = push(cfdic::OP_SET_CIRCULAR, N);
        o.a[0] = cx, o.a[1] = cy, o.a[2] = R;
        copy(o.v[0], W_in);
        copy(o.v[1], W_out);
    }
    // A/sourcecode/allaire_diffuse_io.cpp:312-355
    void set_planar(const double* U_under, const double* U_over, double a, double b, double c) {
        Op& o = push(cfdic::OP_SET_PLANAR);
        o.a[0] = a, o.a[1] = b, o.a[2] = c;
        copy(o.v[0], U_under);
        copy(o.v[1], U_over);
    }
    void set_halfspace(const double* U_under, double a, double b, double c) {
        Op& o = push(cfdic::OP_SET_HALFSPACE);
        o.a[0] = a, o.a[1] = b, o.a[2] = c;
        copy(o.v[0], U_under);
    }
    // W = frac W_in + (1 - frac) W(cell), frac from 10 x 10 sub-samples,
    // cells with frac == 0 untouched.  Unlike add_circle_to_IC this keeps
    // overlapping bubbles physical.
    void blend_circle(const double* W_in, double cx, double cy, double R) {
        Op& o = push(cfdic::OP_BLEND_CIRCLE, 10);
        o.a[0] = cx, o.a[1] = cy, o.a[2] = R;
        copy(o.v[0], W_in);
    }
    void quadrants(const double U[4][4], double xs, double ys) {
        Op& o = push(cfdic::OP_QUADRANTS);
        o.a[0] = xs, o.a[1] = ys;
        for (int k = 0; k < 4; ++k) copy(o.v[k], U[k]);
    }
};

// Fraction of N x N sub-cell sample points of cell (i, j) satisfying inside()
// (E/sourcecode/euler_io.cpp:300-318), for the per-cell Allaire cases.
// E/headers/stiffened_gas_eos.hpp:73-76
double sg_specific_ie(double g, double pinf, double p, double rho) {
    return (p + g * pinf) / ((g - 1.0) * rho);
}

void base_cfg(cfd_config* c, int model, int nx, int ny, int flux_solver) {
    memset(c, 0, sizeof *c);
    c->model = model;
    c->precision = CFD_PREC_FP64;
    c->nx = nx;
    c->ny = ny;
    c->cfl = 0.5;
    c->T = 1.0;
    c->limiter = CFD_LIM_MINMOD;
    c->flux_solver = flux_solver;
    c->splitting = CFD_SPLIT_NAIVE;
    c->wavespeed = CFD_WS_DAVIS;
    c->gamma2 = 1.4;
}

void set_bcs(cfd_config* c, int L, int T, int R, int B) {
    c->bc[CFD_BC_LEFT] = L;
    c->bc[CFD_BC_TOP] = T;
    c->bc[CFD_BC_RIGHT] = R;
    c->bc[CFD_BC_BOTTOM] = B;
}

const int TR = CFD_BC_TRANSMISSIVE, RF = CFD_BC_REFLECTIVE;

// ---------------------------------------------------------------- Euler ---
// E/sourcecode/euler_io.cpp:13-74 (set_parameters)
bool euler_params(const std::string& tc, cfd_config* c) {
    c->gamma1 = 1.4;
    c->pinf1 = 0.0;
    c->x0 = 0.0;
    c->y0 = 0.0;
    c->T = 1.0;
    if (tc == "circular_explosion") {
        c->dx = 2.0 / c->nx;
        c->dy = 2.0 / c->ny;
        set_bcs(c, TR, RF, TR, RF);
    } else if (tc == "multiple_circles_1" || tc == "multiple_circles_2" || tc == "cross" ||
               tc == "internet" || tc == "totem_pole_2") {
        c->dx = 1.0 / c->nx;
        c->dy = 1.0 / c->ny;
        set_bcs(c, TR, TR, TR, TR);
    } else if (tc == "totem_pole_1") {
        c->dx = 1.0 / c->nx;
        c->dy = 1.0 / c->ny;
        set_bcs(c, TR, RF, TR, TR);
    } else if (tc == "totem_pole_3") {
        c->dx = 0.5 / c->nx;
        c->dy = 1.0 / c->ny;
        set_bcs(c, RF, TR, TR, TR);
    } else {
        return false;
    }
    return true;
}

// E/sourcecode/euler_io.cpp:497-726 (initial states)
bool euler_case_program(const std::string& tc, Prog& P, uint64_t seed) {
    auto U_of = [&](double r, double u, double v, double p, double* U) {
        double W[4] = {r, u, v, p};
        cfdic::euler_p2c(P.q, W, U);
    };
    double Ubg[4], Ui[4];
    U_of(0.125, 0.0, 0.0, 0.1, Ubg);
    auto circ = [&](double r, double p, double cx, double cy, double R) {
        U_of(r, 0.0, 0.0, p, Ui);
        P.add_circle(Ui, cx, cy, R);
    };
    auto rect = [&](double r, double p, double bx, double by, double w, double h) {
        U_of(r, 0.0, 0.0, p, Ui);
        P.add_rect(Ui, bx, by, w, h);
    };
    if (tc == "circular_explosion") {
        double Win[4] = {1.0, 0.0, 0.0, 1.0}, Wout[4] = {0.125, 0.0, 0.0, 0.1};
        P.set_circular(Win, Wout, 1.0, 1.0, 0.4, 10);
        return true;
    }
    P.fill(Ubg);
    if (tc == "multiple_circles_1") {
        const double c[9][2] = {{0.5, 0.4}, {0.3, 0.7}, {0.2, 0.7}, {0.6, 0.5}, {0.1, 0.3},
                                {0.3, 0.5}, {0.4, 0.6}, {0.5, 0.4}, {0.5, 0.3}};
        for (auto& p : c) circ(1.0, 1.0, p[0], p[1], 0.1);
    } else if (tc == "multiple_circles_2") {
        circ(1.0, 1.0, 0.0, 0.0, 0.2);
        circ(1.0, 1.0, 0.0, 1.0, 0.2);
        circ(1.0, 1.0, 1.0, 0.0, 0.2);
        circ(1.0, 1.0, 1.0, 1.0, 0.2);
        circ(0.4, 0.0, 0.8, 0.5, 0.1);
        circ(0.3, 0.0, 0.7, 0.5, 0.2);
        circ(0.2, 0.0, 0.6, 0.5, 0.3);
        circ(0.1, 0.0, 0.5, 0.5, 0.4);
    } else if (tc == "cross") {
        circ(1.0, 5.0, 0.0, 0.0, 0.2);
        circ(1.0, 5.0, 0.0, 1.0, 0.2);
        circ(1.0, 5.0, 1.0, 0.0, 0.2);
        circ(1.0, 5.0, 1.0, 1.0, 0.2);
        circ(0.5, 0.0, 0.5, 0.1, 0.11);
        circ(0.5, 0.0, 0.5, 0.9, 0.11);
        circ(0.5, 0.0, 0.3, 0.7, 0.11);
        circ(0.5, 0.0, 0.7, 0.7, 0.11);
        rect(0.5, 0.0, 0.45, 0.1, 0.1, 0.8);
        rect(0.5, 0.0, 0.3, 0.65, 0.4, 0.1);
    } else if (tc == "totem_pole_1") {
        circ(1.0, 5.0, 0.0, 0.0, 0.2);
        circ(1.0, 5.0, 0.0, 1.0, 0.2);
        circ(1.0, 5.0, 1.0, 0.0, 0.2);
        circ(1.0, 5.0, 1.0, 1.0, 0.2);
        rect(0.5, 0.0, 0.45, 0.1, 0.1, 0.8);
        rect(0.5, 0.0, 0.3, 0.65, 0.4, 0.1);
        rect(0.2, 0.0, 0.4, 0.5, 0.2, 0.05);
        rect(0.2, 0.0, 0.4, 0.375, 0.2, 0.075);
        rect(0.2, 0.0, 0.4, 0.25, 0.2, 0.1);
        rect(0.5, 0.0, 0.45, 0.1, 0.1, 0.1);
    } else if (tc == "totem_pole_3") {
        circ(1.0, 5.0, 0.5, 0.0, 0.2);
        circ(1.0, 5.0, 0.5, 1.0, 0.2);
        rect(0.5, 0.0, -0.05, 0.0, 0.1, 0.9);
        rect(0.5, 0.0, -0.2, 0.65, 0.4, 0.1);
        rect(0.2, 0.0, -0.1, 0.5, 0.2, 0.1);
        rect(0.4, 0.0, -0.15, 0.375, 0.3, 0.05);
        rect(0.2, 0.0, -0.1, 0.2, 0.2, 0.1);
        rect(0.5, 0.0, -0.15, 0.0, 0.3, 0.15);
    } else if (tc == "totem_pole_2") {
        circ(1.0, 5.0, 0.0, 0.0, 0.2);
        circ(1.0, 5.0, 0.0, 1.0, 0.2);
        circ(1.0, 5.0, 1.0, 0.0, 0.2);
        circ(1.0, 5.0, 1.0, 1.0, 0.2);
        rect(0.7, 0.0, 0.45, 0.1, 0.1, 0.8);
        rect(0.7, 0.0, 0.3, 0.65, 0.4, 0.1);
        rect(0.4, 0.0, 0.45, 0.575, 0.2, 0.05);
        rect(0.4, 0.0, 0.35, 0.5, 0.2, 0.05);
        rect(0.4, 0.0, 0.4, 0.375, 0.2, 0.075);
        rect(0.4, 0.0, 0.35, 0.25, 0.3, 0.1);
        rect(0.7, 0.0, 0.45, 0.1, 0.1, 0.1);
    } else if (tc == "internet") {
        // The reference seeds from std::random_device (:705-709); here the
        // seed is explicit, the draws are the same engine and distribution.
        int num_people = 16;
        double ddx = 1.0 / num_people;
        std::mt19937 gen((uint32_t)seed);
        std::uniform_real_distribution<> dis(0.0, 1.0);
        for (int i = 0; i < num_people; ++i)
            for (int j = 0; j < num_people; ++j) {
                double cx = (i + 0.5) * ddx + dis(gen) * 0.0;
                double cy = (j + 0.5) * ddx + dis(gen) * 0.0;
                double density = 5.0 * dis(gen);
                circ(density, density, cx, cy, 0.02);
            }
    } else {
        return false;
    }
    return true;
}

// -------------------------------------------------------------- Allaire ---
struct ACase {
    const char* name;
    double g1, g2, p1, p2, x0, y0, Lx, Ly, T;
    int L, Tp, R, B;
};
// A/sourcecode/allaire_diffuse_io.cpp:13-310 (set_parameters)
const ACase kAllaire[] = {
    {"ST1", 1.4, 2.4, 0.0, 0.0, 0.0, 0.0, 1.0, 1.0, 0.14, TR, TR, TR, TR},
    {"ST2", 4.4, 1.4, 600000000.0, 0.0, -2.0, -2.0, 4.0, 4.0, 0.0009, TR, TR, TR, TR},
    {"TTC4", 1.4, 1.4, 0.0, 0.0, 0.0, 0.0, 1.0, 1.0, 0.035, TR, TR, TR, TR},
    {"TTC1", 1.4, 1.4, 0.0, 0.0, 0.0, 0.0, 1.0, 1.0, 0.25, TR, TR, TR, TR},
    {"TTC2", 1.4, 1.4, 0.0, 0.0, 0.0, 0.0, 1.0, 1.0, 0.15, TR, TR, TR, TR},
    {"TTC3", 1.4, 1.4, 0.0, 0.0, 0.0, 0.0, 1.0, 1.0, 0.012, TR, TR, TR, TR},
    {"TTC5", 1.4, 1.4, 0.0, 0.0, 0.0, 0.0, 1.0, 1.0, 0.035, TR, TR, TR, TR},
    {"circular_explosion", 1.4, 1.4, 0.0, 0.0, 0.0, 0.0, 2.0, 2.0, 0.25, TR, TR, TR, TR},
    {"underwater_shocked_bubble", 7.15, 1.4, 3309.0, 0.0, 0.0, 0.0, 12.0, 12.0, 0.05, TR, TR, TR, TR},
    {"underwater_explosion", 1.4, 7.15, 0.0, 3.309e8, -5.0, -5.0, 10.0, 10.0, 0.005, TR, TR, TR, TR},
    {"underwater_explosion_modified", 1.4, 7.15, 0.0, 3.309e8, -5.0, -5.0, 10.0, 10.0, 0.010, TR, RF, TR, RF},
    {"shocked_helium_bubble", 1.4, 1.667, 0.0, 0.0, 0.0, 0.0, 325.0, 89.0, 280.0, TR, RF, TR, RF},
    {"shocked_R22_bubble", 1.4, 1.249, 0.0, 0.0, 0.0, 0.0, 0.445, 0.089, 0.001080, TR, RF, TR, RF},
    {"shocked_SF6", 1.4, 1.076, 0.0, 0.0, 0.0, 0.0, 0.45, 0.2, 0.25, TR, RF, RF, RF},
    {"RMI_SF6", 1.4, 1.093, 0.0, 0.0, 0.0, 0.0, 4.0, 0.5, 10.0, TR, RF, TR, RF},
    {"tin_air_implosion", 3.27, 1.4, 149500.0, 0.0, 0.0, -25.0, 25.0, 50.0, 0.08, RF, TR, TR, TR},
    {"TSTM", 1.5, 1.4, 0.0, 0.0, 0.0, 0.0, 7.0, 3.0, 8.0, TR, TR, TR, TR},
};

const ACase* allaire_lookup(const std::string& tc) {
    std::string key = tc;
    for (const char* suf : {"_x_pure", "_y_pure", "_x", "_y"}) {
        size_t n = strlen(suf);
        if (key.size() > n && key.compare(key.size() - n, n, suf) == 0 &&
            (key.rfind("ST", 0) == 0 || key.rfind("TTC", 0) == 0)) {
            key = key.substr(0, key.size() - n);
            break;
        }
    }
    for (const ACase& c : kAllaire)
        if (key == c.name) return &c;
    return nullptr;
}

// Mixed cell from a volume fraction and two pure-material states
// (A/sourcecode/allaire_diffuse_io.cpp:691-696).
bool allaire_per_cell_case(const std::string& tc) {
    return tc == "shocked_SF6" || tc == "TSTM" || tc == "RMI_SF6" || tc == "tin_air_implosion";
}

// A/sourcecode/allaire_diffuse_io.cpp:402-640 (initial states built from
// the shape helpers)
bool allaire_case_program(const std::string& tc, Prog& P) {
    auto Pc = [&](double a, double b, double c, double d, double e, double f, double* U) {
        double W[6] = {a, b, c, d, e, f};
        cfdic::allaire_p2c(P.q, W, U);
    };
    auto p2c = [&](const double* W, double* U) { cfdic::allaire_p2c(P.q, W, U); };
    double Ul[6], Ur[6];
    bool xdir = tc.find("_x") != std::string::npos;
    auto planar = [&]() {
        if (xdir) P.set_planar(Ul, Ur, 1.0, 0.0, 0.5);
        else P.set_planar(Ul, Ur, 0.0, 1.0, 0.5);
    };
    if (tc == "ST1_x" || tc == "ST1_y") {
        Pc(1.0, 0.0, 0.0, 0.0, 1.0, 1.0, Ul);
        Pc(0.0, 0.125, 0.0, 0.0, 0.1, 0.0, Ur);
        planar();
    } else if (tc == "ST2_x" || tc == "ST2_y") {
        Pc(1000.0, 0.0, 0.0, 0.0, 1000000000.0, 1.0, Ul);
        Pc(0.0, 50.0, 0.0, 0.0, 100000.0, 0.0, Ur);
        if (xdir) P.set_planar(Ul, Ur, 1.0, 0.0, 0.7);
        else P.set_planar(Ul, Ur, 0.0, 1.0, 0.7);
    } else if (tc == "TTC5_x_pure" || tc == "TTC5_y_pure") {
        Pc(5.99924, 0.0, 19.5975, 0.0, 460.894, 1.0, Ul);
        Pc(5.99242, 0.0, -6.19633, 0.0, 46.0950, 1.0, Ur);
        planar();
    } else if (tc == "TTC1_x_pure" || tc == "TTC1_y_pure") {
        Pc(1.0, 0.0, 0.0, 0.0, 1.0, 1.0, Ul);
        Pc(0.125, 0.0, 0.0, 0.0, 0.1, 1.0, Ur);
        planar();
    } else if (tc == "TTC2_x_pure" || tc == "TTC2_y_pure") {
        Pc(1.0, 0.0, -2.0, 0.0, 0.4, 1.0, Ul);
        Pc(1.0, 0.0, 2.0, 0.0, 0.4, 1.0, Ur);
        planar();
    } else if (tc == "TTC3_x_pure" || tc == "TTC3_y_pure") {
        Pc(1.0, 0.0, 0.0, 0.0, 1000.0, 1.0, Ul);
        Pc(1.0, 0.0, 0.0, 0.0, 0.01, 1.0, Ur);
        planar();
    } else if (tc == "TTC4_x_pure" || tc == "TTC4_y_pure") {
        Pc(1.0, 0.0, 0.0, 0.0, 0.1, 1.0, Ul);
        Pc(1.0, 0.0, 0.0, 0.0, 100.0, 1.0, Ur);
        planar();
    } else if (tc == "circular_explosion") {
        double Win[6] = {1.0, 0.0, 0.0, 0.0, 1.0, 1.0}, Wout[6] = {0.0, 0.125, 0.0, 0.0, 0.1, 0.0};
        P.set_circular(Win, Wout, 1.0, 1.0, 0.4, 10);
    } else if (tc == "shocked_helium_bubble") {
        double Wh[6] = {0.0, 0.138, 0.0, 0.0, 1.0, 0.0}, Wpre[6] = {1.0, 0.0, 0.0, 0.0, 1.0, 1.0};
        double Wpost[6] = {1.3764, 0.0, -0.394, 0.0, 1.5698, 1.0};
        P.set_circular(Wh, Wpre, 175.0, 44.5, 25.0, 10);
        p2c(Wpost, Ul);
        P.set_halfspace(Ul, -1.0, 0.0, -225.0);
    } else if (tc == "shocked_R22_bubble") {
        double Wr[6] = {0.0, 3.863, 0.0, 0.0, 1.01325e5, 0.0};
        double Wpre[6] = {1.225, 0.0, 0.0, 0.0, 1.01325e5, 1.0};
        double Wpost[6] = {1.686, 0.0, -113.5, 0.0, 1.59e5, 1.0};
        P.set_circular(Wr, Wpre, 0.225, 0.0445, 0.025, 25);
        p2c(Wpost, Ul);
        P.set_halfspace(Ul, -1.0, 0.0, -0.275);
    } else if (tc == "underwater_shocked_bubble") {
        double Wa[6] = {0.0, 0.0012, 0.0, 0.0, 1.0, 0.0}, Wpre[6] = {1.0, 0.0, 0.0, 0.0, 1.0, 1.0};
        double Wpost[6] = {1.31, 0.0, 67.32, 0.0, 19000.0, 1.0};
        P.set_circular(Wa, Wpre, 6.0, 6.0, 3.0, 10);
        p2c(Wpost, Ul);
        P.set_halfspace(Ul, 1.0, 0.0, 2.4);
    } else if (tc == "underwater_explosion" || tc == "underwater_explosion_modified") {
        double Ww[6] = {0.0, 1000.0, 0.0, 0.0, 1.0e5, 0.0}, Wa[6] = {1.0, 0.0, 0.0, 0.0, 1.0e5, 1.0};
        double Wb[6] = {1270.0, 0.0, 0.0, 0.0, 8.29e8, 1.0};
        P.set_circular(Wb, Ww, 0.0, 0.0, 1.0, 10);
        p2c(Wa, Ul);
        P.set_halfspace(Ul, 0.0, -1.0, -2.5);
    } else {
        return false;
    }
    return true;
}

// A/sourcecode/allaire_diffuse_io.cpp:640-983: the cases whose volume
// fraction comes from a per-cell formula, as MIXED_CELL / RING_CELL
// operations of the shape program (csrc/ic_program.h).
bool allaire_per_cell_program(const std::string& tc, Prog& P) {
    const cfdic::Eos& q = P.q;
    if (tc == "shocked_SF6" || tc == "TSTM" || tc == "RMI_SF6") {
        double rpre, ppre, upre, rpost, ppost, upost, rho2, p2, thr, dir;
        Op& o = P.push(cfdic::OP_MIXED_CELL, 10);
        if (tc == "shocked_SF6") {
            rpre = 1.153; ppre = 9.6856; upre = 0.0;
            rpost = 1.6672; ppost = 16.3256; upost = 1.33273;
            rho2 = 5.805; p2 = 9.6856;
            thr = 0.05; dir = 1.0;  // pre-shock where x > 0.05
            o.v[1][4] = cfdic::REGION_BOX;
            o.a[0] = 0.1, o.a[1] = 0.25, o.a[2] = 0.0, o.a[3] = 0.1;
        } else if (tc == "TSTM") {
            rpre = 0.125; ppre = 0.1; upre = 0.0;
            rpost = 1.0; ppost = 1.0; upost = 0.0;
            rho2 = 1.0; p2 = 0.1;
            thr = 1.0; dir = 1.0;
            o.v[1][4] = cfdic::REGION_BOX;
            o.a[0] = 1.0, o.a[1] = 8.0, o.a[2] = -1.0, o.a[3] = 1.5;
        } else {
            rpre = 1.0; ppre = 1.0; upre = 0.0;
            rpost = 1.411; ppost = 1.628; upost = -0.39;
            rho2 = 5.04; p2 = 1.0;
            thr = 3.2; dir = -1.0;  // pre-shock where x < 3.2
            o.v[1][4] = cfdic::REGION_SINE;
            o.a[0] = std::atan(1.0) * 4.0;
        }
        o.v[0][0] = rpre;
        o.v[0][1] = upre;
        o.v[0][2] = sg_specific_ie(q.g1, q.p1, ppre, rpre);
        o.v[0][3] = rpost;
        o.v[0][4] = upost;
        o.v[0][5] = sg_specific_ie(q.g1, q.p1, ppost, rpost);
        o.v[1][0] = rho2;
        o.v[1][1] = sg_specific_ie(q.g2, q.p2, p2, rho2);
        o.v[1][2] = thr;
        o.v[1][3] = dir;
        return true;
    }
    if (tc == "tin_air_implosion") {
        double rpre = 7.28, ppre = 1.0, rpost = 11.84, ppost = 1000000.0;
        double rho2 = 0.001, p2 = 1.0;
        Op& o = P.push(cfdic::OP_RING_CELL, 10);
        o.v[0][0] = rpre;
        o.v[0][1] = sg_specific_ie(q.g1, q.p1, ppre, rpre);
        o.v[0][2] = rpost;
        o.v[0][3] = sg_specific_ie(q.g1, q.p1, ppost, rpost);
        o.v[1][0] = rho2;
        o.v[1][1] = sg_specific_ie(q.g2, q.p2, p2, rho2);
        o.a[0] = std::atan(1) * 2;
        return true;
    }
    return false;
}

// ------------------------------------------------------------- recipes ---
// Uniform double in [0, 1) from the top 53 bits of a 64-bit Mersenne twister.
struct Rng {
    std::mt19937_64 g;
    explicit Rng(uint64_t s) : g(s) {}
    double u() { return (double)(g() >> 11) * (1.0 / 9007199254740992.0); }
    double range(double a, double b) { return a + (b - a) * u(); }
};

bool recipe_program(const cfd_config* cfg, int recipe, uint64_t seed, int nbubbles, Prog& P) {
    if (recipe == CFD_RECIPE_FOUR_QUADRANT) {
        // 2D Riemann problem split at (0.5, 0.5): quadrants (x>1/2,y>1/2),
        // (x<1/2,y>1/2), (x<1/2,y<1/2), (x>1/2,y<1/2), by cell centre.
        const double Wq[4][4] = {{1.5, 0.0, 0.0, 1.5},
                                 {0.5323, 1.206, 0.0, 0.3},
                                 {0.138, 1.206, 1.206, 0.029},
                                 {0.5323, 0.0, 1.206, 0.3}};
        double Uq[4][4];
        for (int k = 0; k < 4; ++k) cfdic::euler_p2c(P.q, Wq[k], Uq[k]);
        P.quadrants(Uq, 0.5, 0.5);
        return true;
    }
    if (recipe == CFD_RECIPE_SHOCK_BUBBLES) {
        // Background rho = 1, p = 1 at rest; bubbles of log-uniform density
        // at p = 1 blended in; a Mach-2 shock at x = 0.1 moving +x with the
        // Rankine-Hugoniot post-shock state of gamma = 1.4.
        double Wbg[4] = {1.0, 0.0, 0.0, 1.0}, Ubg[4];
        cfdic::euler_p2c(P.q, Wbg, Ubg);
        P.fill(Ubg);
        Rng r(seed);
        for (int b = 0; b < nbubbles; ++b) {
            double cx = r.range(0.2, 1.0), cy = r.u();
            double R = r.range(0.02, 0.08);
            double rho = std::exp(r.range(std::log(0.1), std::log(10.0)));
            double Wb[4] = {rho, 0.0, 0.0, 1.0};
            P.blend_circle(Wb, cx, cy, R);
        }
        double g = cfg->gamma1, M = 2.0;
        double rho2 = (g + 1.0) * M * M / ((g - 1.0) * M * M + 2.0);
        double p2 = 1.0 + 2.0 * g / (g + 1.0) * (M * M - 1.0);
        double u2 = M * std::sqrt(g) * (1.0 - 1.0 / rho2);
        double Wp[4] = {rho2, u2, 0.0, p2}, Up[4];
        cfdic::euler_p2c(P.q, Wp, Up);
        P.set_halfspace(Up, 1.0, 0.0, 0.1);
        return true;
    }
    if (recipe == CFD_RECIPE_WATER_SHOCK_AIR_BUBBLE) {
        // Water (material 1, z = 1 - z_min) at 1e5 Pa with an air bubble
        // (z = z_min) of radius U[0.1, 0.2] centred in [0.6,1.4]x[0.3,0.7];
        // a planar water shock at x = 0.2 with 1e9 Pa behind it and the
        // stiffened-gas Rankine-Hugoniot post-shock state.
        double zm = cfg->z_min > 0.0 ? cfg->z_min : 1e-6;
        double rho_w = 1000.0, rho_a = 1.0, p0 = 1e5, p1 = 1e9;
        Rng r(seed);
        double cx = r.range(0.6, 1.4), cy = r.range(0.3, 0.7), R = r.range(0.1, 0.2);
        double zw = 1.0 - zm, za = zm;
        double Ww[6] = {zw * rho_w, (1.0 - zw) * rho_a, 0.0, 0.0, p0, zw};
        double Wa[6] = {za * rho_w, (1.0 - za) * rho_a, 0.0, 0.0, p0, za};
        P.set_circular(Wa, Ww, cx, cy, R, 10);
        double gw = cfg->gamma1, pi = cfg->pinf1;
        double a1 = p0 + pi, a2 = p1 + pi;
        double ratio = ((gw + 1.0) * a2 + (gw - 1.0) * a1) / ((gw - 1.0) * a2 + (gw + 1.0) * a1);
        double rho_s = rho_w * ratio;
        double u_s = std::sqrt((p1 - p0) * (1.0 / rho_w - 1.0 / rho_s));
        double Ws[6] = {zw * rho_s, (1.0 - zw) * rho_a, u_s, 0.0, p1, zw}, Us[6];
        cfdic::allaire_p2c(P.q, Ws, Us);
        P.set_halfspace(Us, 1.0, 0.0, 0.2);
        return true;
    }
    return false;
}

bool recipe_model_ok(const cfd_config* cfg, int recipe) {
    int want = recipe == CFD_RECIPE_WATER_SHOCK_AIR_BUBBLE ? CFD_MODEL_ALLAIRE : CFD_MODEL_EULER;
    return cfg->model == want;
}

}  // namespace

namespace cfdic {

int case_program(const cfd_config* cfg, const char* test_case, uint64_t seed,
                 std::vector<Op>& ops, Eos& q) {
    if (!cfg || !test_case) return CFD_ERR_INVALID;
    ops.clear();
    q = make_eos(cfg);
    std::string tc = test_case;
    Prog P{q, ops};
    if (cfg->model == CFD_MODEL_EULER) return euler_case_program(tc, P, seed) ? CFD_OK : CFD_ERR_INVALID;
    if (!allaire_lookup(tc)) return CFD_ERR_INVALID;
    if (allaire_per_cell_case(tc)) return allaire_per_cell_program(tc, P) ? CFD_OK : CFD_ERR_INVALID;
    return allaire_case_program(tc, P) ? CFD_OK : CFD_ERR_INVALID;
}

int recipe_program(const cfd_config* cfg, int recipe, uint64_t seed, int nbubbles,
                   std::vector<Op>& ops, Eos& q) {
    if (!cfg) return CFD_ERR_INVALID;
    ops.clear();
    q = make_eos(cfg);
    if (!recipe_model_ok(cfg, recipe)) return CFD_ERR_INVALID;
    Prog P{q, ops};
    return ::recipe_program(cfg, recipe, seed, nbubbles, P) ? CFD_OK : CFD_ERR_INVALID;
}

}  // namespace cfdic

extern "C" {

int cfd_ic_grid_elems(const cfd_config* cfg, size_t* elems) {
    if (!cfg || !elems) return cfd_fail(CFD_ERR_INVALID, "cfd_ic_grid_elems: null argument");
    int g = cfg->flux_solver == CFD_FLUX_GODUNOV ? 1 : 2;
    *elems = (size_t)cfd_nvar(cfg->model) * (cfg->nx + 2 * g) * (size_t)(cfg->ny + 2 * g);
    return CFD_OK;
}

int cfd_case_config(int model, const char* test_case, int nx, int ny, int flux_solver,
                    cfd_config* cfg) {
    if (!test_case || !cfg) return cfd_fail(CFD_ERR_INVALID, "cfd_case_config: null argument");
    if (nx < 2 || ny < 2)
        return cfd_fail(CFD_ERR_INVALID, "grid %dx%d: need at least 2 cells per direction", nx, ny);
    if (model != CFD_MODEL_EULER && model != CFD_MODEL_ALLAIRE)
        return cfd_fail(CFD_ERR_INVALID, "unknown model %d", model);
    base_cfg(cfg, model, nx, ny, flux_solver);
    std::string tc = test_case;
    if (model == CFD_MODEL_EULER) {
        if (euler_params(tc, cfg)) return CFD_OK;
        return cfd_fail(CFD_ERR_INVALID, "unknown Euler test case '%s'", test_case);
    }
    const ACase* a = allaire_lookup(tc);
    if (!a) return cfd_fail(CFD_ERR_INVALID, "unknown Allaire test case '%s'", test_case);
    cfg->gamma1 = a->g1;
    cfg->gamma2 = a->g2;
    cfg->pinf1 = a->p1;
    cfg->pinf2 = a->p2;
    cfg->x0 = a->x0;
    cfg->y0 = a->y0;
    cfg->dx = a->Lx / nx;
    cfg->dy = a->Ly / ny;
    cfg->T = a->T;
    set_bcs(cfg, a->L, a->Tp, a->R, a->B);
    return CFD_OK;
}

int cfd_case_ic(const cfd_config* cfg, const char* test_case, uint64_t seed, double* grid) {
    if (!cfg || !test_case || !grid) return cfd_fail(CFD_ERR_INVALID, "cfd_case_ic: null argument");
    Grid G = make_grid(cfg, grid);
    memset(grid, 0, sizeof(double) * G.nv * G.rows() * G.cols());
    std::vector<Op> ops;
    cfdic::Eos q;
    int r = cfdic::case_program(cfg, test_case, seed, ops, q);
    if (r) return cfd_fail(r, "unknown test case '%s' for model %d", test_case, cfg->model);
    run_program(G, ops, q);
    return CFD_OK;
}

int cfd_recipe_config(int recipe, int nx, int ny, cfd_config* cfg) {
    if (!cfg) return cfd_fail(CFD_ERR_INVALID, "cfd_recipe_config: null argument");
    if (nx < 2 || ny < 2)
        return cfd_fail(CFD_ERR_INVALID, "grid %dx%d: need at least 2 cells per direction", nx, ny);
    switch (recipe) {
        case CFD_RECIPE_FOUR_QUADRANT:
            base_cfg(cfg, CFD_MODEL_EULER, nx, ny, CFD_FLUX_MUSCL);
            cfg->gamma1 = 1.4;
            cfg->dx = 1.0 / nx;
            cfg->dy = 1.0 / ny;
            cfg->cfl = 0.8;
            cfg->T = 0.3;
            cfg->limiter = CFD_LIM_VANLEER;
            set_bcs(cfg, TR, TR, TR, TR);
            return CFD_OK;
        case CFD_RECIPE_SHOCK_BUBBLES:
            base_cfg(cfg, CFD_MODEL_EULER, nx, ny, CFD_FLUX_MUSCL);
            cfg->gamma1 = 1.4;
            cfg->dx = 1.0 / nx;
            cfg->dy = 1.0 / ny;
            cfg->cfl = 0.8;
            cfg->T = INFINITY;
            set_bcs(cfg, TR, RF, TR, RF);
            return CFD_OK;
        case CFD_RECIPE_WATER_SHOCK_AIR_BUBBLE:
            base_cfg(cfg, CFD_MODEL_ALLAIRE, nx, ny, CFD_FLUX_MUSCL);
            cfg->gamma1 = 4.4;
            cfg->pinf1 = 6e8;
            cfg->gamma2 = 1.4;
            cfg->pinf2 = 0.0;
            cfg->dx = 2.0 / nx;
            cfg->dy = 1.0 / ny;
            cfg->cfl = 0.6;
            cfg->T = INFINITY;
            cfg->wavespeed = CFD_WS_PVRS;
            cfg->z_min = 1e-6;
            set_bcs(cfg, TR, TR, TR, TR);
            return CFD_OK;
    }
    return cfd_fail(CFD_ERR_INVALID, "unknown recipe %d", recipe);
}

int cfd_recipe_ic(const cfd_config* cfg, int recipe, uint64_t seed, int nbubbles, double* grid) {
    if (!cfg || !grid) return cfd_fail(CFD_ERR_INVALID, "cfd_recipe_ic: null argument");
    Grid G = make_grid(cfg, grid);
    std::vector<Op> ops;
    cfdic::Eos q;
    int r = cfdic::recipe_program(cfg, recipe, seed, nbubbles, ops, q);
    if (r) return cfd_fail(r, "recipe %d does not apply to this configuration (model %d)", recipe,
                           cfg->model);
    run_program(G, ops, q);
    return CFD_OK;
}

}  // extern "C"
