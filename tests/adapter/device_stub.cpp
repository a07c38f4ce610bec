// TEST INFRASTRUCTURE ONLY.  Stand-ins for the device entry points of the C
// ABI that the reference-loop adapter (cfd-art_b200/adapter/gpu_problem.hpp)
// calls, computed by the CPU oracle (oracle/cfd_oracle.c), so that the
// adapter's call sequence -- which call takes the step, when the state is
// read back, where the masses go -- can be checked against the reference's
// own output files on a machine without a GPU.  Linked only into the test
// binary oracle/_ref/ref_main_stub_*; the library never contains it, and the
// adapter linked against the real library (oracle/_ref/ref_main_gpu_*) fails
// with CFD_ERR_CUDA where no device exists.
//
// The stub keeps the reference's two grids with their ghost cells (the
// oracle's buffer semantics), so CFD_LAYOUT_GHOSTED_AOS_AS_REFERENCE is the
// oracle's grid as it stands.  cfd_step can only take the step that the
// oracle's own dt rule gives; any other dt is refused.
#include <cstdarg>
#include <cstdio>
#include <cstring>
#include <vector>

#include "cfd_oracle.h"
#include "cfdgpu.h"

struct cfd_solver {
    cfd_config cfg;
    ref_params p;
    int model = 0, g = 2, nv = 4;
    bool ref_ghosts = false, uploaded = false;
    std::vector<double> grid, future;
    int n = 0;
    double t = 0.0, mass[2] = {0.0, 0.0};
};

static thread_local char g_err[512];

static int stub_fail(int code, const char* fmt, ...) {
    va_list ap;
    va_start(ap, fmt);
    std::vsnprintf(g_err, sizeof g_err, fmt, ap);
    va_end(ap);
    return code;
}

extern "C" {

int cfd_last_error(char* buf, size_t len) {
    if (buf && len) {
        std::strncpy(buf, g_err, len - 1);
        buf[len - 1] = '\0';
    }
    return (int)std::strlen(g_err);
}

int cfd_create(const cfd_config* cfg, cfd_solver** out) {
    if (!cfg || !out) return stub_fail(CFD_ERR_INVALID, "null argument");
    if (cfg->precision != CFD_PREC_FP64) return stub_fail(CFD_ERR_UNSUPPORTED, "stub: FP64 only");
    cfd_solver* s = new cfd_solver;
    s->cfg = *cfg;
    s->model = cfg->model == CFD_MODEL_EULER ? ORACLE_EULER : ORACLE_ALLAIRE;
    s->nv = cfg->model == CFD_MODEL_EULER ? 4 : 6;
    s->g = cfg->flux_solver == CFD_FLUX_GODUNOV ? 1 : 2;
    ref_params& p = s->p;
    std::memset(&p, 0, sizeof p);
    p.nx = cfg->nx;
    p.ny = cfg->ny;
    p.x0 = cfg->x0;
    p.y0 = cfg->y0;
    p.dx = cfg->dx;
    p.dy = cfg->dy;
    p.gamma1 = cfg->gamma1;
    p.pinf1 = cfg->pinf1;
    p.gamma2 = cfg->gamma2;
    p.pinf2 = cfg->pinf2;
    for (int k = 0; k < 4; ++k) p.bc[k] = cfg->bc[k];  // same L, R, B, T order and codes
    p.cfl = cfg->cfl;
    p.T = cfg->T;
    p.limiter = cfg->limiter;
    p.flux_solver = cfg->flux_solver;
    p.splitting = cfg->splitting;
    p.wavespeed = cfg->wavespeed;
    p.z_min = cfg->z_min;
    p.fix_dy_halfstep = cfg->fix_dy_halfstep;
    *out = s;
    return CFD_OK;
}

int cfd_destroy(cfd_solver* s) {
    delete s;
    return CFD_OK;
}

int cfd_nvar(int model) { return model == CFD_MODEL_ALLAIRE ? 6 : 4; }

int cfd_set_reference_ghosts(cfd_solver* s, int enable) {
    if (!s) return stub_fail(CFD_ERR_INVALID, "null solver");
    s->ref_ghosts = enable != 0;
    return CFD_OK;
}

int cfd_upload(cfd_solver* s, const double* host, int layout, int n, double t) {
    if (!s || !host) return stub_fail(CFD_ERR_INVALID, "null argument");
    if (layout != CFD_LAYOUT_GHOSTED_AOS) return stub_fail(CFD_ERR_UNSUPPORTED, "stub layout");
    size_t elems = (size_t)(s->p.ny + 2 * s->g) * (s->p.nx + 2 * s->g) * s->nv;
    s->grid.assign(host, host + elems);
    s->future = s->grid;
    s->n = n;
    s->t = t;
    s->uploaded = true;
    return CFD_OK;
}

int cfd_compute_dt(cfd_solver* s, int n, double t, double* dt_out) {
    if (!s || !dt_out) return stub_fail(CFD_ERR_INVALID, "null argument");
    if (!s->uploaded) return stub_fail(CFD_ERR_STATE, "compute_dt before upload");
    *dt_out = oracle_compute_dt(s->model, &s->p, s->grid.data(), n, t, s->mass);
    return CFD_OK;
}

int cfd_get_status(cfd_solver* s, cfd_status* st) {
    if (!s || !st) return stub_fail(CFD_ERR_INVALID, "null argument");
    std::memset(st, 0, sizeof *st);
    st->n = s->n;
    st->t = s->t;
    st->done = s->t >= s->p.T;
    st->mass1 = s->mass[0];
    st->mass2 = s->mass[1];
    return CFD_OK;
}

int cfd_step(cfd_solver* s, double dt) {
    if (!s) return stub_fail(CFD_ERR_INVALID, "null solver");
    if (!s->uploaded) return stub_fail(CFD_ERR_STATE, "step before upload");
    double taken_dt = 0.0;
    int taken = oracle_run(s->model, &s->p, s->grid.data(), s->future.data(), 1, &s->n, &s->t,
                           &taken_dt);
    if (taken != 1 || taken_dt != dt)
        return stub_fail(CFD_ERR_STATE, "stub: asked for dt %.17g, the oracle's rule gives %.17g",
                         dt, taken_dt);
    return CFD_OK;
}

int cfd_download(cfd_solver* s, double* host, int layout) {
    if (!s || !host) return stub_fail(CFD_ERR_INVALID, "null argument");
    if (layout != CFD_LAYOUT_GHOSTED_AOS_AS_REFERENCE || !s->ref_ghosts)
        return stub_fail(CFD_ERR_UNSUPPORTED, "stub: reference-ghost downloads only");
    std::memcpy(host, s->grid.data(), s->grid.size() * sizeof(double));
    return CFD_OK;
}

}  // extern "C"
