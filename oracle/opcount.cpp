// Operation counter for the plain-C restatement (cfd_oracle.c).  TEST AND
// MEASUREMENT INFRASTRUCTURE ONLY: never linked into the shipped library.
//
// cfd_oracle.c is compiled a second time, as C++, with every `double` it
// declares replaced by `opc::fp`, a double that counts the arithmetic done on
// it.  The arithmetic itself is unchanged (each operator performs the same
// IEEE operation on the wrapped value, compiled with -ffp-contract=off), so a
// counted run returns bit-identical states to the plain build, which the
// tests check.  The count is exact for the input given: MUSCL-Hancock's
// fallbacks, the limiter's branches, the PVRS choice and the Euler fix-ups
// are data dependent, so a figure always belongs to a stated workload.
//
// Categories (OPC_*): additions and subtractions, multiplications,
// divisions, square roots, comparisons (every <, <=, >, >=, == of two values,
// which includes the min/max selections), and fabs/copysign.  Negation is a
// sign flip and is not counted.  Operations between two literal constants are
// folded by the compiler in both the reference and this file and are not
// counted either.
//
// Phases: compute_dt (E/sourcecode/euler_timestep.cpp:7-44,
// A/sourcecode/allaire_diffuse_timestep.cpp:8-48) and the split step with
// its boundary fills (E/headers/splitting_scheme.hpp:37-67, :78-122).
#include <math.h>
#include <stdint.h>
#include <stdlib.h>
#include <string.h>

#include "cfd_oracle.h"

namespace opc {

enum { ADD = 0, MUL, DIV, SQRT, CMP, SIGN, NCAT };
enum { PH_DT = 0, PH_STEP, PH_OTHER, NPH };

static uint64_t counts[NPH][NCAT];
static int phase = PH_OTHER;

struct fp {
    double v;
    fp() = default;
    fp(double x) : v(x) {}
    explicit operator double() const { return v; }
    fp& operator+=(fp o) { ++counts[phase][ADD]; v = v + o.v; return *this; }
    fp& operator-=(fp o) { ++counts[phase][ADD]; v = v - o.v; return *this; }
    fp& operator*=(fp o) { ++counts[phase][MUL]; v = v * o.v; return *this; }
    fp& operator/=(fp o) { ++counts[phase][DIV]; v = v / o.v; return *this; }
};

inline fp operator+(fp a, fp b) { ++counts[phase][ADD]; return fp(a.v + b.v); }
inline fp operator-(fp a, fp b) { ++counts[phase][ADD]; return fp(a.v - b.v); }
inline fp operator*(fp a, fp b) { ++counts[phase][MUL]; return fp(a.v * b.v); }
inline fp operator/(fp a, fp b) { ++counts[phase][DIV]; return fp(a.v / b.v); }
inline fp operator-(fp a) { return fp(-a.v); }
inline bool operator<(fp a, fp b) { ++counts[phase][CMP]; return a.v < b.v; }
inline bool operator<=(fp a, fp b) { ++counts[phase][CMP]; return a.v <= b.v; }
inline bool operator>(fp a, fp b) { ++counts[phase][CMP]; return a.v > b.v; }
inline bool operator>=(fp a, fp b) { ++counts[phase][CMP]; return a.v >= b.v; }
inline bool operator==(fp a, fp b) { ++counts[phase][CMP]; return a.v == b.v; }

}  // namespace opc

// Found by ordinary lookup from the restatement's calls (the libm overloads
// take plain doubles, to which opc::fp does not convert implicitly).
static inline opc::fp sqrt(opc::fp a) {
    ++opc::counts[opc::phase][opc::SQRT];
    return opc::fp(::sqrt(a.v));
}
static inline opc::fp fabs(opc::fp a) {
    ++opc::counts[opc::phase][opc::SIGN];
    return opc::fp(::fabs(a.v));
}
static inline opc::fp copysign(opc::fp a, opc::fp b) {
    ++opc::counts[opc::phase][opc::SIGN];
    return opc::fp(::copysign(a.v, b.v));
}

// The restatement's exported names are taken by the plain build's header
// (already included above, with plain doubles); the counted definitions get
// their own names.
#define oracle_run opc_counted_oracle_run
#define oracle_compute_dt opc_counted_oracle_compute_dt
#define oracle_face_flux opc_counted_oracle_face_flux
#define double opc::fp
#include "cfd_oracle.c"
#undef double
#undef oracle_run
#undef oracle_compute_dt
#undef oracle_face_flux

namespace {

void reset() { memset(opc::counts, 0, sizeof(opc::counts)); }

void copy_counts(uint64_t* out) {
    for (int ph = 0; ph < opc::NPH; ++ph)
        for (int c = 0; c < opc::NCAT; ++c) out[ph * opc::NCAT + c] = opc::counts[ph][c];
}

}  // namespace

extern "C" {

// Number of categories and phases of the count arrays below (row-major
// [phase][category], phases dt, step, other).
int opcount_layout(int* n_categories, int* n_phases) {
    *n_categories = opc::NCAT;
    *n_phases = opc::NPH;
    return 0;
}

// The time loop of oracle_run (headers/simulation.hpp:48-61 with the step
// stop), counted.  `grid` holds the ghosted AoS state and is advanced in
// place; `counts` receives NPH * NCAT totals for the whole run.
int opcount_run(int model, const ref_params* p, double* grid, int max_steps, int* n_io,
                double* t_io, uint64_t* counts) {
    static_assert(sizeof(opc::fp) == sizeof(double), "opc::fp must be layout-compatible");
    reset();
    eosp q = make_eos(model, p);
    grid_t G, F;
    G.nx = F.nx = p->nx;
    G.ny = F.ny = p->ny;
    G.g = F.g = p->flux_solver == REF_FLUX_GODUNOV ? 1 : 2;
    G.rows = F.rows = G.ny + 2 * G.g;
    G.cols = F.cols = G.nx + 2 * G.g;
    G.nv = F.nv = q.nv;
    size_t bytes = sizeof(double) * (size_t)G.rows * G.cols * G.nv;
    opc::fp* A = static_cast<opc::fp*>(malloc(bytes));
    opc::fp* B = static_cast<opc::fp*>(malloc(bytes));
    if (!A || !B) {
        free(A);
        free(B);
        return -1;
    }
    memcpy(A, grid, bytes);
    memcpy(B, grid, bytes);
    G.a = A;
    F.a = B;
    int n = *n_io, taken = 0;
    double t = *t_io;
    while (t < p->T && taken < max_steps) {
        opc::phase = opc::PH_DT;
        double dt = static_cast<double>(compute_dt(&q, p, &G, n, t, NULL));
        opc::phase = opc::PH_STEP;
        advance(&q, p, &G, &F, dt);
        opc::phase = opc::PH_OTHER;
        t += dt;
        n++;
        taken++;
        if (::fabs(t - p->T) < 1e-12) t = p->T;
    }
    memcpy(grid, G.a, bytes);
    free(A);
    free(B);
    *n_io = n;
    *t_io = t;
    copy_counts(counts);
    return taken;
}

// One face of the flux solver (MUSCL-Hancock or Godunov), counted.
void opcount_face(int model, const ref_params* p, const double* stencil, double dt, double dx,
                  double* flux, double* u_star, double* z_star, uint64_t* counts) {
    reset();
    eosp q = make_eos(model, p);
    opc::fp us = 0.0, zs = 0.0;
    opc::phase = opc::PH_STEP;
    face_flux(&q, p, reinterpret_cast<const opc::fp*>(stencil), dt, dx,
              reinterpret_cast<opc::fp*>(flux), &us, &zs);
    opc::phase = opc::PH_OTHER;
    *u_star = us.v;
    if (z_star) *z_star = zs.v;
    copy_counts(counts);
}

}  // extern "C"
