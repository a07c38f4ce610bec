// C ABI of the B200 split finite-volume solver: solver objects, device
// memory, layout conversion and launch of the sweep kernels.  Compiled with
// --fmad=false (see __graft_entry__.build) like the kernels it instantiates.
#include <cuda_runtime.h>

#include <algorithm>
#include <cmath>
#include <cstdarg>
#include <cstdio>
#include <cstring>
#include <map>
#include <mutex>
#include <new>
#include <string>
#include <utility>
#include <vector>

#include "../../include/cfdgpu.h"
#include "cfd_checkpoint.h"
#include "cfd_config.h"
#include "cfd_error.h"
#include "cfd_frame.h"
#include "cfd_ic.h"
#include "cfd_pool.h"
#include "cfd_sweep.cuh"
#include "ic_builders.h"

using namespace cfd;

namespace {
thread_local std::string g_err;
}

namespace cfd {

cudaError_t pool_alloc(void** p, size_t bytes, cudaStream_t stream) {
    static std::mutex mu;
    static std::map<int, cudaMemPool_t> pools;
    int dev = 0;
    cudaError_t e = cudaGetDevice(&dev);
    if (e) return e;
    cudaMemPool_t pool;
    {
        std::lock_guard<std::mutex> lk(mu);
        auto it = pools.find(dev);
        if (it == pools.end()) {
            cudaMemPoolProps props;
            memset(&props, 0, sizeof props);
            props.allocType = cudaMemAllocationTypePinned;
            props.location.type = cudaMemLocationTypeDevice;
            props.location.id = dev;
            if ((e = cudaMemPoolCreate(&pool, &props))) return e;
            unsigned long long keep = ~0ULL;  // keep released blocks for reuse
            if ((e = cudaMemPoolSetAttribute(pool, cudaMemPoolAttrReleaseThreshold, &keep)))
                return e;
            pools[dev] = pool;
        } else {
            pool = it->second;
        }
    }
    return cudaMallocFromPoolAsync(p, bytes, pool, stream);
}

cudaError_t pool_free(void* p, cudaStream_t stream) {
    return p ? cudaFreeAsync(p, stream) : cudaSuccess;
}

}  // namespace cfd

// Records the message cfd_last_error() returns on this thread.
int cfd_fail(int code, const char* fmt, ...) {
    char buf[512];
    va_list ap;
    va_start(ap, fmt);
    vsnprintf(buf, sizeof buf, fmt, ap);
    va_end(ap);
    g_err = buf;
    return code;
}

namespace {

#define fail cfd_fail

#define CUDA_TRY(expr)                                                                   \
    do {                                                                                 \
        cudaError_t e_ = (expr);                                                         \
        if (e_ != cudaSuccess)                                                           \
            return fail(e_ == cudaErrorMemoryAllocation ? CFD_ERR_NOMEM : CFD_ERR_CUDA,  \
                        "%s: %s (%s:%d)", #expr, cudaGetErrorString(e_), __FILE__, __LINE__); \
    } while (0)

// Tile shapes: x-sweep 64 cells along x by 4 rows; y-sweep 32 cells along y
// by 8 columns.
constexpr int TSX = 60, NAX = 4, TSY = 28, NAY = 8;

int round_up(int v, int m) { return (v + m - 1) / m * m; }

}  // namespace

struct cfd_solver {
    cfd_config cfg;
    int nv = 4, g = 2;
    int pitch = 0;
    long long plane = 0;
    size_t buf_elems = 0;
    double* buf[2] = {nullptr, nullptr};
    DevState* dst = nullptr;
    double* partials = nullptr;
    int max_blocks = 0;
    unsigned long long* counters = nullptr;
    cudaStream_t stream = nullptr;
    bool own_stream = false;
    bool uploaded = false;
    Eos eos;
    cudaGraphExec_t graph = nullptr;
    int graph_steps = 0;
    // reference ghost values (cfd_set_reference_ghosts): the ghost frame
    double* frame = nullptr;
    bool ref_ghosts = false;
    // kernel timing: event pairs around each sweep launch, by sweep direction
    bool timing = false;
    std::vector<std::pair<cudaEvent_t, cudaEvent_t>> ev[2];
    double ev_ms[2] = {0.0, 0.0};
    int ev_n[2] = {0, 0};
};

namespace cfd {

// cfd_create's checks of a configuration (cfd_config.h).
int validate_config(const cfd_config* c) {
    if (!c) return fail(CFD_ERR_INVALID, "null config");
    if (c->model != CFD_MODEL_EULER && c->model != CFD_MODEL_ALLAIRE)
        return fail(CFD_ERR_INVALID, "unknown model %d", c->model);
    if (c->precision != CFD_PREC_FP64 && c->precision != CFD_PREC_MIXED &&
        c->precision != CFD_PREC_FP64_FAST)
        return fail(CFD_ERR_INVALID, "unknown precision %d", c->precision);
    if (c->precision != CFD_PREC_FP64)
        return fail(CFD_ERR_UNSUPPORTED,
                    "a single solver is the bit-identical FP64 form; the mixed and fast FP64 "
                    "forms run as batch members (cfd_batch_add) or through the server");
    if (c->nx < 2 || c->ny < 2)
        return fail(CFD_ERR_INVALID, "grid %dx%d: need at least 2 cells per direction", c->nx,
                    c->ny);
    if ((long long)c->nx * c->ny > (1LL << 31))
        return fail(CFD_ERR_INVALID, "grid %dx%d too large", c->nx, c->ny);
    if (!(c->dx > 0.0) || !(c->dy > 0.0)) return fail(CFD_ERR_INVALID, "dx, dy must be > 0");
    if (!(c->gamma1 > 1.0)) return fail(CFD_ERR_INVALID, "gamma1 must be > 1");
    if (c->model == CFD_MODEL_ALLAIRE && !(c->gamma2 > 1.0))
        return fail(CFD_ERR_INVALID, "gamma2 must be > 1");
    for (int k = 0; k < 4; ++k)
        if (c->bc[k] != CFD_BC_TRANSMISSIVE && c->bc[k] != CFD_BC_REFLECTIVE)
            return fail(CFD_ERR_INVALID, "bad boundary condition %d on side %d", c->bc[k], k);
    if (c->limiter < 0 || c->limiter > 3) return fail(CFD_ERR_INVALID, "bad limiter");
    if (c->flux_solver != CFD_FLUX_MUSCL && c->flux_solver != CFD_FLUX_GODUNOV)
        return fail(CFD_ERR_INVALID, "bad flux solver");
    if (c->splitting != CFD_SPLIT_NAIVE && c->splitting != CFD_SPLIT_STRANG)
        return fail(CFD_ERR_INVALID, "bad splitting scheme");
    if (c->wavespeed != CFD_WS_DAVIS && c->wavespeed != CFD_WS_PVRS)
        return fail(CFD_ERR_INVALID, "bad wave-speed estimate");
    if (!(c->z_min >= 0.0 && c->z_min < 0.5)) return fail(CFD_ERR_INVALID, "z_min in [0, 0.5)");
    if (!(c->cfl > 0.0)) return fail(CFD_ERR_INVALID, "cfl must be > 0");
    return CFD_OK;
}

Eos make_eos(const cfd_config& c) {
    Eos q;
    q.g1 = c.gamma1;
    q.p1 = c.pinf1;
    q.g2 = c.model == CFD_MODEL_ALLAIRE ? c.gamma2 : 1.4;
    q.p2 = c.model == CFD_MODEL_ALLAIRE ? c.pinf2 : 0.0;
    q.gm1_1 = q.g1 - 1.0;
    q.gm1_2 = q.g2 - 1.0;
    q.gp1 = q.g1 * q.p1;
    return q;
}

}  // namespace cfd

namespace {

void layout_sizes(const cfd_config& c, int& nv, int& g, int& pitch, long long& plane,
                  size_t& buf_elems) {
    nv = c.model == CFD_MODEL_EULER ? 4 : 6;
    g = c.flux_solver == CFD_FLUX_GODUNOV ? 1 : 2;
    pitch = round_up(c.nx, 32);
    plane = (long long)round_up(c.ny, 1) * pitch;
    size_t soa = (size_t)nv * plane;
    size_t ghosted = (size_t)nv * (c.nx + 2 * g) * (size_t)(c.ny + 2 * g);
    buf_elems = std::max(soa, ghosted);
    buf_elems = (buf_elems + 31) / 32 * 32;
}

int sweep_blocks(const cfd_config& c, int dir) {
    if (dir == DIR_X) return ((c.nx + TSX - 1) / TSX) * ((c.ny + NAX - 1) / NAX);
    return ((c.ny + TSY - 1) / TSY) * ((c.nx + NAY - 1) / NAY);
}

template <int MODEL, int DIR, int TS, int NA>
int launch_sweep_t(const SweepArgs& a, int blocks, cudaStream_t st) {
    constexpr int smem = sweep_smem_bytes<MODEL, DIR, TS, NA>();
    static bool attr_set = false;
    if (!attr_set) {
        CUDA_TRY(cudaFuncSetAttribute(sweep_kernel<MODEL, DIR, TS, NA>,
                                      cudaFuncAttributeMaxDynamicSharedMemorySize, smem));
        attr_set = true;
    }
    sweep_kernel<MODEL, DIR, TS, NA><<<blocks, 256, smem, st>>>(a);
    CUDA_TRY(cudaGetLastError());
    return CFD_OK;
}

int launch_sweep(int model, int dir, const SweepArgs& a, int blocks, cudaStream_t st) {
    if (model == CFD_MODEL_EULER)
        return dir == DIR_X ? launch_sweep_t<MODEL_EULER, DIR_X, TSX, NAX>(a, blocks, st)
                            : launch_sweep_t<MODEL_EULER, DIR_Y, TSY, NAY>(a, blocks, st);
    return dir == DIR_X ? launch_sweep_t<MODEL_ALLAIRE, DIR_X, TSX, NAX>(a, blocks, st)
                        : launch_sweep_t<MODEL_ALLAIRE, DIR_Y, TSY, NAY>(a, blocks, st);
}

// Kernel arguments of one sweep reading bufs[cur ^ in_sel] and writing the
// other buffer, where cur is the device-side index of the current state.
SweepArgs sweep_args(cfd_solver* s, int dir, int in_sel, double dt_scale, bool host_dt, double dt,
                     bool reduce, bool flip) {
    const cfd_config& c = s->cfg;
    SweepArgs a;
    a.bufs[0] = s->buf[0];
    a.bufs[1] = s->buf[1];
    a.in_sel = in_sel;
    a.flip_cur = flip ? 1 : 0;
    a.plane = s->plane;
    a.pitch = s->pitch;
    a.nx = c.nx;
    a.ny = c.ny;
    a.eos = s->eos;
    if (dir == DIR_X) {
        a.bc_lo = c.bc[CFD_BC_LEFT];
        a.bc_hi = c.bc[CFD_BC_RIGHT];
        a.h_flux = c.dx;
        a.h_upd = c.dx;
    } else {
        a.bc_lo = c.bc[CFD_BC_BOTTOM];
        a.bc_hi = c.bc[CFD_BC_TOP];
        a.h_flux = c.fix_dy_halfstep ? c.dy : c.dx;  // reference quirk: params.dx
        a.h_upd = c.dy;
    }
    a.limiter = c.limiter;
    a.wavespeed = c.wavespeed;
    a.godunov = c.flux_solver == CFD_FLUX_GODUNOV;
    a.z_min = c.z_min;
    a.dt_host = dt;
    a.dt_scale = dt_scale;
    a.use_host_dt = host_dt ? 1 : 0;
    a.reduce = reduce ? 1 : 0;
    a.advance_time = reduce ? 1 : 0;
    a.st = s->dst;
    a.partials = s->partials;
    a.counters = s->counters;
    return a;
}

int timed_sweep(cfd_solver* s, int dir, const SweepArgs& a, int blocks) {
    if (!s->timing) return launch_sweep(s->cfg.model, dir, a, blocks, s->stream);
    cudaEvent_t e0, e1;
    CUDA_TRY(cudaEventCreate(&e0));
    CUDA_TRY(cudaEventCreate(&e1));
    CUDA_TRY(cudaEventRecord(e0, s->stream));
    int r = launch_sweep(s->cfg.model, dir, a, blocks, s->stream);
    CUDA_TRY(cudaEventRecord(e1, s->stream));
    s->ev[dir].emplace_back(e0, e1);
    return r;
}

// One split step (E/headers/splitting_scheme.hpp:37-67 naive, :78-122 Strang).
// Naive: x cur -> other, y other -> cur.  Strang: x/2 cur -> other,
// y other -> cur, x/2 cur -> other, and the last sweep flips cur.  The
// buffer roles are resolved on the device, so a step skipped because t >= T
// leaves them untouched.
int enqueue_frame_snapshot(cfd_solver* s, int in_sel, bool host_dt);

int enqueue_step(cfd_solver* s, bool host_dt, double dt) {
    const cfd_config& c = s->cfg;
    int bx = sweep_blocks(c, DIR_X), by = sweep_blocks(c, DIR_Y);
    int r;
    // reference ghost values: the buffer current after the step keeps the
    // fill made before the sweep that read it last (naive: the x sweep;
    // Strang: the y sweep)
    if (c.splitting == CFD_SPLIT_NAIVE) {
        if (s->ref_ghosts && (r = enqueue_frame_snapshot(s, 0, host_dt))) return r;
        SweepArgs ax = sweep_args(s, DIR_X, 0, 1.0, host_dt, dt, false, false);
        if ((r = timed_sweep(s, DIR_X, ax, bx))) return r;
        SweepArgs ay = sweep_args(s, DIR_Y, 1, 1.0, host_dt, dt, true, false);
        return timed_sweep(s, DIR_Y, ay, by);
    }
    SweepArgs a1 = sweep_args(s, DIR_X, 0, 0.5, host_dt, dt, false, false);
    if ((r = timed_sweep(s, DIR_X, a1, bx))) return r;
    if (s->ref_ghosts && (r = enqueue_frame_snapshot(s, 1, host_dt))) return r;
    SweepArgs a2 = sweep_args(s, DIR_Y, 1, 1.0, host_dt, dt, false, false);
    if ((r = timed_sweep(s, DIR_Y, a2, by))) return r;
    SweepArgs a3 = sweep_args(s, DIR_X, 0, 0.5, host_dt, dt, true, true);
    return timed_sweep(s, DIR_X, a3, bx);
}

// ---- layout conversion and the initial reduction ---------------------------

__global__ void ghosted_to_soa(const double* __restrict__ src, double* __restrict__ dst, int nx,
                               int ny, int g, int nv, int pitch, long long plane) {
    long long n = (long long)nx * ny;
    for (long long idx = blockIdx.x * (long long)blockDim.x + threadIdx.x; idx < n;
         idx += (long long)gridDim.x * blockDim.x) {
        int i = (int)(idx / nx), j = (int)(idx % nx);
        const double* c = src + ((long long)(i + g) * (nx + 2 * g) + (j + g)) * nv;
        for (int k = 0; k < nv; ++k) dst[k * plane + (long long)i * pitch + j] = c[k];
    }
}

// Interior plus the boundary fill of pre_sweep (E/sourcecode/euler_ppsweep.cpp:7-118)
// of the current state; corner ghosts are left zero (never filled or read).
__global__ void soa_to_ghosted(const double* __restrict__ src, double* __restrict__ dst, int nx,
                               int ny, int g, int nv, int pitch, long long plane, int bcL, int bcR,
                               int bcB, int bcT, int im, int it) {
    int W = nx + 2 * g, H = ny + 2 * g;
    long long n = (long long)W * H;
    for (long long idx = blockIdx.x * (long long)blockDim.x + threadIdx.x; idx < n;
         idx += (long long)gridDim.x * blockDim.x) {
        int gi = (int)(idx / W), gj = (int)(idx % W);
        int i = gi - g, j = gj - g;
        double* d = dst + idx * nv;
        bool ri = i >= 0 && i < ny, rj = j >= 0 && j < nx;
        if (!ri && !rj) {
            for (int k = 0; k < nv; ++k) d[k] = 0.0;
            continue;
        }
        int si = i, sj = j, neg = -1;
        if (j < 0) { sj = -j - 1; if (bcL) neg = im; }
        else if (j >= nx) { sj = 2 * nx - 1 - j; if (bcR) neg = im; }
        if (i < 0) { si = -i - 1; if (bcB) neg = it; }
        else if (i >= ny) { si = 2 * ny - 1 - i; if (bcT) neg = it; }
        for (int k = 0; k < nv; ++k) {
            double v = src[k * plane + (long long)si * pitch + sj];
            d[k] = (k == neg) ? -v : v;
        }
    }
}

// ---- schlieren field -------------------------------------------------------
// |grad rho| by central differences at every interior cell, as the
// reference's writer forms it (E/sourcecode/euler_io.cpp:1142-1185,
// A/sourcecode/allaire_diffuse_io.cpp:1109-1150): gx = (rho_r - rho_l) /
// (2 dx), gy = (rho_t - rho_b) / (2 dy), sqrt(gx^2 + gy^2), every operation
// correctly rounded and none contracted, so the values equal the host
// writer's.  An edge cell's outside neighbour is the boundary fill of the
// current state (a mirror: the density of the edge cell itself) or, with
// `frame`, the reference's ghost value.  Output row-major from the bottom
// row, nx x ny.
template <int MODEL>
__device__ __forceinline__ double sch_rho(const double* __restrict__ src, long long plane,
                                          long long off) {
    return MODEL == MODEL_EULER ? src[off] : src[off] + src[plane + off];
}

template <int MODEL>
__device__ __forceinline__ double sch_frame_rho(const double* __restrict__ frame, int gi, int gj,
                                                int nx, int ny, int g, int nv) {
    const double* fr = frame + frame_index(gi, gj, nx, ny, g) * nv;
    return MODEL == MODEL_EULER ? fr[0] : fr[0] + fr[1];
}

template <int MODEL>
__global__ void schlieren_field(const double* __restrict__ src, const double* __restrict__ frame,
                                double* __restrict__ out, int nx, int ny, int g, int nv,
                                int pitch, long long plane, double dx, double dy) {
    const long long n = (long long)nx * ny;
    for (long long idx = blockIdx.x * (long long)blockDim.x + threadIdx.x; idx < n;
         idx += (long long)gridDim.x * blockDim.x) {
        const int i = (int)(idx / nx), j = (int)(idx % nx);
        const long long o = (long long)i * pitch + j;
        const double rc = sch_rho<MODEL>(src, plane, o);
        double rl, rr, rb, rt;
        if (j > 0) rl = sch_rho<MODEL>(src, plane, o - 1);
        else rl = frame ? sch_frame_rho<MODEL>(frame, i + g, g - 1, nx, ny, g, nv) : rc;
        if (j < nx - 1) rr = sch_rho<MODEL>(src, plane, o + 1);
        else rr = frame ? sch_frame_rho<MODEL>(frame, i + g, nx + g, nx, ny, g, nv) : rc;
        if (i > 0) rb = sch_rho<MODEL>(src, plane, o - pitch);
        else rb = frame ? sch_frame_rho<MODEL>(frame, g - 1, j + g, nx, ny, g, nv) : rc;
        if (i < ny - 1) rt = sch_rho<MODEL>(src, plane, o + pitch);
        else rt = frame ? sch_frame_rho<MODEL>(frame, ny + g, j + g, nx, ny, g, nv) : rc;
        const double gx = (rr - rl) / (2.0 * dx);
        const double gy = (rt - rb) / (2.0 * dy);
        out[idx] = sqrt(gx * gx + gy * gy);
    }
}

// ---- reference ghost values --------------------------------------------------
// The reference's grid keeps its ghost cells between boundary fills: after
// set_ICs they hold the initial condition's own values, later the fill that
// pre_sweep (E/sourcecode/euler_ppsweep.cpp:7-118) made before the last sweep
// that read the buffer, and the corners are never refilled.  The solver keeps
// those values in a ghost frame (cfd_frame.h) when asked to.

// Every ghost cell (corners included) of a ghosted AoS grid.
__global__ void frame_from_ghosted(const double* __restrict__ src, double* __restrict__ frame,
                                   int nx, int ny, int g, int nv) {
    const long long n = frame_cells(nx, ny, g);
    for (long long f = blockIdx.x * (long long)blockDim.x + threadIdx.x; f < n;
         f += (long long)gridDim.x * blockDim.x) {
        int gi, gj;
        frame_cell(f, nx, ny, g, gi, gj);
        const double* c = src + ((long long)gi * (nx + 2 * g) + gj) * nv;
        for (int k = 0; k < nv; ++k) frame[f * nv + k] = c[k];
    }
}

// The boundary fill of the sweep input bufs[cur ^ in_sel] into the frame's
// edge cells (corners untouched), skipped like the sweeps once the device
// time loop is done.
__global__ void frame_snapshot(const double* __restrict__ b0, const double* __restrict__ b1, int in_sel, const DevState* st,
                               int use_host_dt, double* __restrict__ frame, int nx, int ny, int g,
                               int nv, int pitch, long long plane, int bcL, int bcR, int bcB,
                               int bcT, int im, int it) {
    if (!use_host_dt && st->done) return;
    const double* __restrict__ src = ((st->cur ^ in_sel) & 1) ? b1 : b0;
    const long long n = frame_cells(nx, ny, g);
    for (long long f = blockIdx.x * (long long)blockDim.x + threadIdx.x; f < n;
         f += (long long)gridDim.x * blockDim.x) {
        int gi, gj;
        frame_cell(f, nx, ny, g, gi, gj);
        const int i = gi - g, j = gj - g;
        const bool ri = i >= 0 && i < ny, rj = j >= 0 && j < nx;
        if (!ri && !rj) continue;  // corner
        int si = i, sj = j, neg = -1;
        if (j < 0) { sj = -j - 1; if (bcL) neg = im; }
        else if (j >= nx) { sj = 2 * nx - 1 - j; if (bcR) neg = im; }
        if (i < 0) { si = -i - 1; if (bcB) neg = it; }
        else if (i >= ny) { si = 2 * ny - 1 - i; if (bcT) neg = it; }
        for (int k = 0; k < nv; ++k) {
            double v = src[k * plane + (long long)si * pitch + sj];
            frame[f * nv + k] = (k == neg) ? -v : v;
        }
    }
}

// Interior from the SoA state, ghost cells from the frame.
__global__ void soa_frame_to_ghosted(const double* __restrict__ src,
                                     const double* __restrict__ frame, double* __restrict__ dst,
                                     int nx, int ny, int g, int nv, int pitch, long long plane) {
    int W = nx + 2 * g, H = ny + 2 * g;
    long long n = (long long)W * H;
    for (long long idx = blockIdx.x * (long long)blockDim.x + threadIdx.x; idx < n;
         idx += (long long)gridDim.x * blockDim.x) {
        int gi = (int)(idx / W), gj = (int)(idx % W);
        int i = gi - g, j = gj - g;
        double* d = dst + idx * nv;
        if (i >= 0 && i < ny && j >= 0 && j < nx) {
            for (int k = 0; k < nv; ++k) d[k] = src[k * plane + (long long)i * pitch + j];
        } else {
            const double* fr = frame + frame_index(gi, gj, nx, ny, g) * nv;
            for (int k = 0; k < nv; ++k) d[k] = fr[k];
        }
    }
}

int enqueue_frame_snapshot(cfd_solver* s, int in_sel, bool host_dt) {
    const cfd_config& c = s->cfg;
    int im = c.model == CFD_MODEL_EULER ? 1 : 2;
    frame_snapshot<<<148, 256, 0, s->stream>>>(
        s->buf[0], s->buf[1], in_sel, s->dst, host_dt ? 1 : 0, s->frame, c.nx, c.ny, s->g, s->nv,
        s->pitch, s->plane, c.bc[CFD_BC_LEFT], c.bc[CFD_BC_RIGHT], c.bc[CFD_BC_BOTTOM],
        c.bc[CFD_BC_TOP], im, im + 1);
    CUDA_TRY(cudaGetLastError());
    return CFD_OK;
}

template <int MODEL>
__global__ void reduce_state(const double* __restrict__ in, long long plane, int pitch, int nx,
                             int ny, Eos q, DevState* st, double* partials) {
    constexpr int NV = ModelTraits<MODEL>::NV;
    double r_mu = 0.0, r_mv = 0.0, r_m1 = 0.0, r_m2 = 0.0;
    long long n = (long long)nx * ny;
    for (long long idx = blockIdx.x * (long long)blockDim.x + threadIdx.x; idx < n;
         idx += (long long)gridDim.x * blockDim.x) {
        int i = (int)(idx / nx), j = (int)(idx % nx);
        double U[NV];
        for (int k = 0; k < NV; ++k) U[k] = in[k * plane + (long long)i * pitch + j];
        double su, sv, m1, m2;
        wave_speeds<MODEL>(q, U, su, sv, m1, m2);
        r_mu = smax(r_mu, su);
        r_mv = smax(r_mv, sv);
        r_m1 += m1;
        r_m2 += m2;
    }
    __shared__ double red[4][32];
    __shared__ bool is_last;
    for (int o = 16; o > 0; o >>= 1) {
        r_mu = smax(r_mu, __shfl_down_sync(0xffffffffu, r_mu, o));
        r_mv = smax(r_mv, __shfl_down_sync(0xffffffffu, r_mv, o));
        r_m1 += __shfl_down_sync(0xffffffffu, r_m1, o);
        r_m2 += __shfl_down_sync(0xffffffffu, r_m2, o);
    }
    if ((threadIdx.x & 31) == 0) {
        red[0][threadIdx.x >> 5] = r_mu;
        red[1][threadIdx.x >> 5] = r_mv;
        red[2][threadIdx.x >> 5] = r_m1;
        red[3][threadIdx.x >> 5] = r_m2;
    }
    __syncthreads();
    if (threadIdx.x == 0) {
        double mu = red[0][0], mv = red[1][0], m1 = red[2][0], m2 = red[3][0];
        for (int w = 1; w < (int)(blockDim.x >> 5); ++w) {
            mu = smax(mu, red[0][w]);
            mv = smax(mv, red[1][w]);
            m1 += red[2][w];
            m2 += red[3][w];
        }
        double* p = partials + 4 * blockIdx.x;
        p[0] = mu;
        p[1] = mv;
        p[2] = m1;
        p[3] = m2;
        __threadfence();
        unsigned t = atomicAdd(&st->ticket, 1u);
        is_last = (t == gridDim.x - 1);
    }
    __syncthreads();
    if (is_last) {
        __threadfence();
        finish_reduction(st, partials, gridDim.x, 0, 0.0, 0);
    }
}

int enqueue_reduce(cfd_solver* s) {
    int blocks = std::min(s->max_blocks, 148 * 4);
    long long n = (long long)s->cfg.nx * s->cfg.ny;
    blocks = (int)std::max(1LL, std::min<long long>(blocks, (n + 255) / 256));
    if (s->cfg.model == CFD_MODEL_EULER)
        reduce_state<MODEL_EULER><<<blocks, 256, 0, s->stream>>>(
            s->buf[0], s->plane, s->pitch, s->cfg.nx, s->cfg.ny, s->eos, s->dst, s->partials);
    else
        reduce_state<MODEL_ALLAIRE><<<blocks, 256, 0, s->stream>>>(
            s->buf[0], s->plane, s->pitch, s->cfg.nx, s->cfg.ny, s->eos, s->dst, s->partials);
    CUDA_TRY(cudaGetLastError());
    return CFD_OK;
}

// ---- single-face test kernel ----------------------------------------------
// The same P2/P3 logic as the sweep, for one face from a 4-cell stencil.
template <int MODEL>
__global__ void face_flux_kernel(int nfaces, const double* __restrict__ st, Eos q, int limiter,
                                 int wavespeed, int godunov, double z_min, double s_half,
                                 double* flux, double* ustar, double* zstar) {
    constexpr int NV = ModelTraits<MODEL>::NV;
    int f = blockIdx.x * blockDim.x + threadIdx.x;
    if (f >= nfaces) return;
    const int m = godunov ? 2 : 4;
    const double* S = st + (size_t)f * m * NV;
    double EL[NV], ER[NV];
    if (godunov) {
        for (int k = 0; k < NV; ++k) {
            EL[k] = S[k];
            ER[k] = S[NV + k];
        }
    } else {
        Prim<MODEL> P[4];
        for (int c = 0; c < 4; ++c) cons_to_prim<MODEL>(q, S + c * NV, P[c]);
        // cell 1 -> high-face states, cell 2 -> low-face states
        double Ep[NV], Em[NV];
        unsigned fl1 = 0, fl2 = 0;
        for (int side = 0; side < 2; ++side) {
            int c = 1 + side;
            double d[NV], Wt[NV], Ut[NV], e, X[NV];
            for (int k = 0; k < NV; ++k)
                d[k] = limit1(limiter, P[c].W[k] - P[c - 1].W[k], P[c + 1].W[k] - P[c].W[k]);
            unsigned fl = 0;
            for (int k = 0; k < NV; ++k) Wt[k] = P[c].W[k] + 0.5 * d[k];
            prim_to_cons<MODEL>(q, Wt, Ut, e);
            if (muscl_check<MODEL>(Ut, Wt, e)) fl |= 1u;
            for (int k = 0; k < NV; ++k) Wt[k] = P[c].W[k] - 0.5 * d[k];
            prim_to_cons<MODEL>(q, Wt, Ut, e);
            if (muscl_check<MODEL>(Ut, Wt, e)) fl |= 2u;
            jacobian_times<MODEL>(q, P[c], d, s_half, X);
            if (side == 0) {
                for (int k = 0; k < NV; ++k) Wt[k] = (P[c].W[k] + 0.5 * d[k]) - X[k];
                prim_to_cons<MODEL>(q, Wt, Ep, e);
                if (muscl_check<MODEL>(Ep, Wt, e)) fl |= 4u;
                fl1 = fl;
            } else {
                for (int k = 0; k < NV; ++k) Wt[k] = (P[c].W[k] - 0.5 * d[k]) - X[k];
                prim_to_cons<MODEL>(q, Wt, Em, e);
                if (muscl_check<MODEL>(Em, Wt, e)) fl |= 8u;
                fl2 = fl;
            }
        }
        bool ok2;
        if ((fl1 & 1u) && (fl2 & 2u)) {
            for (int k = 0; k < NV; ++k) {
                EL[k] = Ep[k];
                ER[k] = Em[k];
            }
            ok2 = (fl1 & 4u) && (fl2 & 8u);
        } else {
            double Wt[NV], e;
            zero_slope_state<MODEL>(q, P[1], s_half, true, Wt);
            prim_to_cons<MODEL>(q, Wt, EL, e);
            bool okL = muscl_check<MODEL>(EL, Wt, e);
            zero_slope_state<MODEL>(q, P[2], s_half, false, Wt);
            prim_to_cons<MODEL>(q, Wt, ER, e);
            bool okR = muscl_check<MODEL>(ER, Wt, e);
            ok2 = okL && okR;
        }
        if (!ok2) {
            for (int k = 0; k < NV; ++k) {
                EL[k] = S[NV + k];
                ER[k] = S[2 * NV + k];
            }
        }
    }
    double F[NV], us;
    hllc_flux<MODEL>(q, wavespeed, EL, ER, F, us);
    for (int k = 0; k < NV; ++k) flux[(size_t)f * NV + k] = F[k];
    ustar[f] = us;
    if (MODEL == MODEL_ALLAIRE && zstar) {
        double cs = copysign(1.0, us);
        zstar[f] = godunov ? (((1.0 + cs) / 2.0) * EL[5]) + (((1.0 - cs) / 2.0) * ER[5])
                           : ((0.5 * (1.0 + cs)) * EL[5]) + ((0.5 * (1.0 - cs)) * ER[5]);
    }
    (void)z_min;
}

}  // namespace

// ============================================================== C ABI ======

extern "C" {

const char* cfd_version(void) { return "cfdgpu 0.1 (sm_100a, FP64 split FV)"; }

int cfd_last_error(char* buf, size_t len) {
    if (buf && len) {
        strncpy(buf, g_err.c_str(), len - 1);
        buf[len - 1] = 0;
    }
    return (int)g_err.size();
}

int cfd_nvar(int model) { return model == CFD_MODEL_ALLAIRE ? 6 : 4; }

int cfd_device_bytes(const cfd_config* cfg, size_t* bytes) {
    int r = validate_config(cfg);
    if (r) return r;
    int nv, g, pitch;
    long long plane;
    size_t be;
    layout_sizes(*cfg, nv, g, pitch, plane, be);
    int mb = std::max(sweep_blocks(*cfg, DIR_X), sweep_blocks(*cfg, DIR_Y));
    *bytes = 2 * be * sizeof(double) + sizeof(DevState) + 4 * sizeof(double) * mb +
             CNT_N * sizeof(unsigned long long);
    return CFD_OK;
}

int cfd_create(const cfd_config* cfg, cfd_solver** out) {
    if (!out) return fail(CFD_ERR_INVALID, "null output pointer");
    *out = nullptr;
    int r = validate_config(cfg);
    if (r) return r;
    int ndev = 0;
    if (cudaGetDeviceCount(&ndev) != cudaSuccess || ndev == 0)
        return fail(CFD_ERR_CUDA, "no CUDA device available");
    cfd_solver* s = new (std::nothrow) cfd_solver();
    if (!s) return fail(CFD_ERR_NOMEM, "host allocation failed");
    s->cfg = *cfg;
    s->eos = make_eos(*cfg);
    layout_sizes(*cfg, s->nv, s->g, s->pitch, s->plane, s->buf_elems);
    s->max_blocks = std::max({sweep_blocks(*cfg, DIR_X), sweep_blocks(*cfg, DIR_Y), 148 * 4});
    auto cleanup = [&](int code) {
        cfd_destroy(s);
        return code;
    };
    cudaError_t e;
    if (cfg->stream) {
        s->stream = (cudaStream_t)cfg->stream;
    } else {
        if ((e = cudaStreamCreateWithFlags(&s->stream, cudaStreamNonBlocking)) != cudaSuccess)
            return cleanup(fail(CFD_ERR_CUDA, "stream creation failed: %s", cudaGetErrorString(e)));
        s->own_stream = true;
    }
    // stream-ordered allocations: no device-wide synchronisation while other
    // solves run (a server creates and destroys solves between their rounds)
    auto alloc = [&](void** p, size_t bytes) { return pool_alloc(p, bytes, s->stream); };
    for (int b = 0; b < 2; ++b) {
        e = alloc(reinterpret_cast<void**>(&s->buf[b]), s->buf_elems * sizeof(double));
        if (e != cudaSuccess)
            return cleanup(fail(CFD_ERR_NOMEM, "device allocation of %zu bytes failed: %s",
                                s->buf_elems * sizeof(double), cudaGetErrorString(e)));
    }
    if ((e = alloc(reinterpret_cast<void**>(&s->dst), sizeof(DevState))) != cudaSuccess ||
        (e = alloc(reinterpret_cast<void**>(&s->partials), 4 * sizeof(double) * s->max_blocks)) !=
            cudaSuccess ||
        (e = alloc(reinterpret_cast<void**>(&s->counters), CNT_N * sizeof(unsigned long long))) !=
            cudaSuccess)
        return cleanup(fail(CFD_ERR_NOMEM, "device allocation failed: %s", cudaGetErrorString(e)));
    DevState init;
    memset(&init, 0, sizeof init);
    init.T = cfg->T;
    init.cfl = cfg->cfl;
    init.dx = cfg->dx;
    init.dy = cfg->dy;
    if ((e = cudaMemcpyAsync(s->dst, &init, sizeof init, cudaMemcpyHostToDevice, s->stream)) !=
            cudaSuccess ||
        (e = cudaMemsetAsync(s->counters, 0, CNT_N * sizeof(unsigned long long), s->stream)) !=
            cudaSuccess)
        return cleanup(fail(CFD_ERR_CUDA, "initialisation failed: %s", cudaGetErrorString(e)));
    *out = s;
    return CFD_OK;
}

int cfd_destroy(cfd_solver* s) {
    if (!s) return CFD_OK;
    if (s->stream) cudaStreamSynchronize(s->stream);
    if (s->graph) cudaGraphExecDestroy(s->graph);
    for (int d = 0; d < 2; ++d)
        for (auto& pr : s->ev[d]) {
            cudaEventDestroy(pr.first);
            cudaEventDestroy(pr.second);
        }
    if (s->stream) {
        pool_free(s->buf[0], s->stream);
        pool_free(s->buf[1], s->stream);
        pool_free(s->dst, s->stream);
        pool_free(s->partials, s->stream);
        pool_free(s->counters, s->stream);
    }
    if (s->frame) cudaFree(s->frame);
    if (s->own_stream && s->stream) cudaStreamDestroy(s->stream);
    delete s;
    return CFD_OK;
}

static int set_time(cfd_solver* s, int n, double t) {
    DevState init;
    memset(&init, 0, sizeof init);
    init.T = s->cfg.T;
    init.cfl = s->cfg.cfl;
    init.dx = s->cfg.dx;
    init.dy = s->cfg.dy;
    init.n = n;
    init.t = t;
    CUDA_TRY(cudaMemcpyAsync(s->dst, &init, sizeof init, cudaMemcpyHostToDevice, s->stream));
    // pageable source: the copy is complete when the call returns
    return CFD_OK;
}

// Ghost frame of a state uploaded without ghost values: the boundary fill of
// the current state, corners zero.
static int frame_from_state(cfd_solver* s) {
    const cfd_config& c = s->cfg;
    CUDA_TRY(cudaMemsetAsync(s->frame, 0,
                             sizeof(double) * s->nv * frame_cells(c.nx, c.ny, s->g), s->stream));
    return enqueue_frame_snapshot(s, 0, true);
}

int cfd_upload(cfd_solver* s, const double* host, int layout, int n, double t) {
    if (!s || !host) return fail(CFD_ERR_INVALID, "null argument");
    const cfd_config& c = s->cfg;
    int r;
    if (layout == CFD_LAYOUT_GHOSTED_AOS) {
        size_t elems = (size_t)s->nv * (c.nx + 2 * s->g) * (size_t)(c.ny + 2 * s->g);
        CUDA_TRY(cudaMemcpyAsync(s->buf[1], host, elems * sizeof(double), cudaMemcpyHostToDevice,
                                 s->stream));
        ghosted_to_soa<<<148 * 8, 256, 0, s->stream>>>(s->buf[1], s->buf[0], c.nx, c.ny, s->g,
                                                       s->nv, s->pitch, s->plane);
        CUDA_TRY(cudaGetLastError());
        if (s->frame) {
            frame_from_ghosted<<<148, 256, 0, s->stream>>>(s->buf[1], s->frame, c.nx, c.ny, s->g,
                                                           s->nv);
            CUDA_TRY(cudaGetLastError());
        }
    } else if (layout == CFD_LAYOUT_SOA) {
        for (int k = 0; k < s->nv; ++k)
            CUDA_TRY(cudaMemcpy2DAsync(s->buf[0] + k * s->plane, s->pitch * sizeof(double),
                                       host + (size_t)k * c.nx * c.ny, c.nx * sizeof(double),
                                       c.nx * sizeof(double), c.ny, cudaMemcpyHostToDevice,
                                       s->stream));
    } else {
        return fail(CFD_ERR_INVALID, "unknown layout %d", layout);
    }
    if ((r = set_time(s, n, t))) return r;
    if (s->frame && layout != CFD_LAYOUT_GHOSTED_AOS && (r = frame_from_state(s))) return r;
    if ((r = enqueue_reduce(s))) return r;
    s->uploaded = true;
    return CFD_OK;
}

int cfd_upload_device(cfd_solver* s, const double* dev, int n, double t) {
    if (!s || !dev) return fail(CFD_ERR_INVALID, "null argument");
    const cfd_config& c = s->cfg;
    for (int k = 0; k < s->nv; ++k)
        CUDA_TRY(cudaMemcpy2DAsync(s->buf[0] + k * s->plane, s->pitch * sizeof(double),
                                   dev + (size_t)k * c.nx * c.ny, c.nx * sizeof(double),
                                   c.nx * sizeof(double), c.ny, cudaMemcpyDeviceToDevice,
                                   s->stream));
    int r;
    if ((r = set_time(s, n, t))) return r;
    if (s->frame && (r = frame_from_state(s))) return r;
    if ((r = enqueue_reduce(s))) return r;
    s->uploaded = true;
    return CFD_OK;
}

// Builds a shape program's state on the device in the solver's first
// buffer, then sets the time and reduces the wave speeds as cfd_upload does.
static int upload_program(cfd_solver* s, const std::vector<cfdic::Op>& ops, const cfdic::Eos& q,
                          int n, double t) {
    const cfd_config& c = s->cfg;
    cfdic::Geom geo{c.x0, c.y0, c.dx, c.dy};
    CUDA_TRY(cfdic::build_device(ops, q, geo, c.nx, c.ny, s->buf[0], s->plane, s->pitch,
                                 s->stream));
    if (s->frame)
        CUDA_TRY(cfdic::build_frame_device(ops, q, geo, c.nx, c.ny, s->g, s->frame, s->stream));
    int r;
    if ((r = set_time(s, n, t))) return r;
    if ((r = enqueue_reduce(s))) return r;
    s->uploaded = true;
    return CFD_OK;
}

int cfd_upload_recipe(cfd_solver* s, int recipe, uint64_t seed, int nbubbles, int n, double t) {
    if (!s) return fail(CFD_ERR_INVALID, "null argument");
    std::vector<cfdic::Op> ops;
    cfdic::Eos q;
    int r = cfdic::recipe_program(&s->cfg, recipe, seed, nbubbles, ops, q);
    if (r) return fail(r, "recipe %d does not apply to this configuration", recipe);
    return upload_program(s, ops, q, n, t);
}

int cfd_upload_case(cfd_solver* s, const char* test_case, uint64_t seed, int n, double t) {
    if (!s || !test_case) return fail(CFD_ERR_INVALID, "null argument");
    std::vector<cfdic::Op> ops;
    cfdic::Eos q;
    int r = cfdic::case_program(&s->cfg, test_case, seed, ops, q);
    if (r) return fail(r, "unknown test case %s", test_case);
    return upload_program(s, ops, q, n, t);
}

static int current_buffer(cfd_solver* s, int& cur) {
    DevState d;
    CUDA_TRY(cudaMemcpyAsync(&d, s->dst, sizeof d, cudaMemcpyDeviceToHost, s->stream));
    CUDA_TRY(cudaStreamSynchronize(s->stream));
    cur = d.cur & 1;
    return CFD_OK;
}

int cfd_download(cfd_solver* s, double* host, int layout) {
    if (!s || !host) return fail(CFD_ERR_INVALID, "null argument");
    if (!s->uploaded) return fail(CFD_ERR_STATE, "no state uploaded");
    const cfd_config& c = s->cfg;
    int cur, r;
    if ((r = current_buffer(s, cur))) return r;
    double* src = s->buf[cur];
    double* scratch = s->buf[cur ^ 1];
    if (layout == CFD_LAYOUT_GHOSTED_AOS) {
        int im = c.model == CFD_MODEL_EULER ? 1 : 2;
        soa_to_ghosted<<<148 * 8, 256, 0, s->stream>>>(
            src, scratch, c.nx, c.ny, s->g, s->nv, s->pitch, s->plane, c.bc[0], c.bc[1],
            c.bc[2], c.bc[3], im, im + 1);
        CUDA_TRY(cudaGetLastError());
        size_t elems = (size_t)s->nv * (c.nx + 2 * s->g) * (size_t)(c.ny + 2 * s->g);
        CUDA_TRY(cudaMemcpyAsync(host, scratch, elems * sizeof(double), cudaMemcpyDeviceToHost,
                                 s->stream));
    } else if (layout == CFD_LAYOUT_GHOSTED_AOS_AS_REFERENCE) {
        if (!s->frame)
            return fail(CFD_ERR_STATE, "reference ghost values are off (cfd_set_reference_ghosts)");
        soa_frame_to_ghosted<<<148 * 8, 256, 0, s->stream>>>(src, s->frame, scratch, c.nx, c.ny,
                                                             s->g, s->nv, s->pitch, s->plane);
        CUDA_TRY(cudaGetLastError());
        size_t elems = (size_t)s->nv * (c.nx + 2 * s->g) * (size_t)(c.ny + 2 * s->g);
        CUDA_TRY(cudaMemcpyAsync(host, scratch, elems * sizeof(double), cudaMemcpyDeviceToHost,
                                 s->stream));
    } else if (layout == CFD_LAYOUT_SOA) {
        for (int k = 0; k < s->nv; ++k)
            CUDA_TRY(cudaMemcpy2DAsync(host + (size_t)k * c.nx * c.ny, c.nx * sizeof(double),
                                       src + k * s->plane, s->pitch * sizeof(double),
                                       c.nx * sizeof(double), c.ny, cudaMemcpyDeviceToHost,
                                       s->stream));
    } else {
        return fail(CFD_ERR_INVALID, "unknown layout %d", layout);
    }
    CUDA_TRY(cudaStreamSynchronize(s->stream));
    return CFD_OK;
}

int cfd_schlieren(cfd_solver* s, int ghosts, double* host) {
    if (!s || !host) return fail(CFD_ERR_INVALID, "null argument");
    if (!s->uploaded) return fail(CFD_ERR_STATE, "no state uploaded");
    if (ghosts != CFD_LAYOUT_GHOSTED_AOS && ghosts != CFD_LAYOUT_GHOSTED_AOS_AS_REFERENCE)
        return fail(CFD_ERR_INVALID, "ghosts: CFD_LAYOUT_GHOSTED_AOS or _AS_REFERENCE");
    const double* frame = nullptr;
    if (ghosts == CFD_LAYOUT_GHOSTED_AOS_AS_REFERENCE) {
        if (!s->frame)
            return fail(CFD_ERR_STATE, "reference ghost values are off (cfd_set_reference_ghosts)");
        frame = s->frame;
    }
    const cfd_config& c = s->cfg;
    int cur, r;
    if ((r = current_buffer(s, cur))) return r;
    double* out = s->buf[cur ^ 1];  // scratch: the other state buffer
    if (c.model == CFD_MODEL_EULER)
        schlieren_field<MODEL_EULER><<<148 * 8, 256, 0, s->stream>>>(
            s->buf[cur], frame, out, c.nx, c.ny, s->g, s->nv, s->pitch, s->plane, c.dx, c.dy);
    else
        schlieren_field<MODEL_ALLAIRE><<<148 * 8, 256, 0, s->stream>>>(
            s->buf[cur], frame, out, c.nx, c.ny, s->g, s->nv, s->pitch, s->plane, c.dx, c.dy);
    CUDA_TRY(cudaGetLastError());
    CUDA_TRY(cudaMemcpyAsync(host, out, sizeof(double) * c.nx * (size_t)c.ny,
                             cudaMemcpyDeviceToHost, s->stream));
    CUDA_TRY(cudaStreamSynchronize(s->stream));
    return CFD_OK;
}

int cfd_get_status(cfd_solver* s, cfd_status* out) {
    if (!s || !out) return fail(CFD_ERR_INVALID, "null argument");
    DevState d;
    CUDA_TRY(cudaMemcpyAsync(&d, s->dst, sizeof d, cudaMemcpyDeviceToHost, s->stream));
    CUDA_TRY(cudaMemcpyAsync(out->counters, s->counters, sizeof out->counters,
                             cudaMemcpyDeviceToHost, s->stream));
    CUDA_TRY(cudaStreamSynchronize(s->stream));
    out->n = d.n;
    out->done = d.done;
    out->t = d.t;
    out->dt_next = d.dt;
    out->maxu = d.maxu;
    out->maxv = d.maxv;
    out->mass1 = d.mass1;
    out->mass2 = d.mass2;
    return CFD_OK;
}

int cfd_compute_dt(cfd_solver* s, int n, double t, double* dt_out) {
    if (!s || !dt_out) return fail(CFD_ERR_INVALID, "null argument");
    if (!s->uploaded) return fail(CFD_ERR_STATE, "no state uploaded");
    DevState d;
    CUDA_TRY(cudaMemcpyAsync(&d, s->dst, sizeof d, cudaMemcpyDeviceToHost, s->stream));
    CUDA_TRY(cudaStreamSynchronize(s->stream));
    // E/sourcecode/euler_timestep.cpp:36-43 on the reduced wave speeds
    double cfl = s->cfg.cfl;
    if (n < 5) cfl = (0.2 < cfl) ? 0.2 : cfl;
    double a = s->cfg.dx / d.maxu, b = s->cfg.dy / d.maxv;
    double dt = cfl * ((b < a) ? b : a);
    if (t + dt > s->cfg.T) dt = s->cfg.T - t;
    *dt_out = dt;
    return CFD_OK;
}

int cfd_step(cfd_solver* s, double dt) {
    if (!s) return fail(CFD_ERR_INVALID, "null solver");
    if (!s->uploaded) return fail(CFD_ERR_STATE, "no state uploaded");
    return enqueue_step(s, true, dt);
}

int cfd_advance(cfd_solver* s, int max_steps) {
    if (!s) return fail(CFD_ERR_INVALID, "null solver");
    if (!s->uploaded) return fail(CFD_ERR_STATE, "no state uploaded");
    if (max_steps < 0) return fail(CFD_ERR_INVALID, "negative step count");
    // Chunks of 16 steps replay one captured CUDA graph; the rest launch directly.
    const int K = 16;
    int r;
    if (s->timing) {
        for (int i = 0; i < max_steps; ++i)
            if ((r = enqueue_step(s, false, 0.0))) return r;
        return CFD_OK;
    }
    if (max_steps >= K) {
        if (!s->graph) {
            cudaStream_t cap = s->stream;
            CUDA_TRY(cudaStreamBeginCapture(cap, cudaStreamCaptureModeThreadLocal));
            int rr = CFD_OK;
            for (int i = 0; i < K && rr == CFD_OK; ++i) rr = enqueue_step(s, false, 0.0);
            cudaGraph_t gph;
            cudaError_t e = cudaStreamEndCapture(cap, &gph);
            if (rr) return rr;
            if (e != cudaSuccess) return fail(CFD_ERR_CUDA, "capture: %s", cudaGetErrorString(e));
            e = cudaGraphInstantiate(&s->graph, gph, 0);
            cudaGraphDestroy(gph);
            if (e != cudaSuccess)
                return fail(CFD_ERR_CUDA, "graph instantiate: %s", cudaGetErrorString(e));
            s->graph_steps = K;
        }
        for (int i = 0; i + K <= max_steps; i += K) CUDA_TRY(cudaGraphLaunch(s->graph, s->stream));
    }
    for (int i = 0; i < max_steps % K; ++i)
        if ((r = enqueue_step(s, false, 0.0))) return r;
    return CFD_OK;
}

// ---- checkpoint / resume --------------------------------------------------

int cfd_checkpoint_save(cfd_solver* s, const char* path) {
    if (!s || !path) return fail(CFD_ERR_INVALID, "null argument");
    if (!s->uploaded) return fail(CFD_ERR_STATE, "no state uploaded");
    const cfd_config& c = s->cfg;
    DevState d;
    CkptHeader h;
    ckpt_init(h);
    CUDA_TRY(cudaMemcpyAsync(&d, s->dst, sizeof d, cudaMemcpyDeviceToHost, s->stream));
    CUDA_TRY(cudaMemcpyAsync(h.counters, s->counters, sizeof h.counters, cudaMemcpyDeviceToHost,
                             s->stream));
    CUDA_TRY(cudaStreamSynchronize(s->stream));
    h.cfg = c;
    h.cfg.stream = nullptr;
    h.nv = s->nv;
    h.g = s->g;
    h.n = d.n;
    h.done = d.done;
    h.t = d.t;
    h.dt = d.dt;
    h.maxu = d.maxu;
    h.maxv = d.maxv;
    h.mass1 = d.mass1;
    h.mass2 = d.mass2;
    h.has_frame = s->frame != nullptr;
    const size_t cells = (size_t)c.nx * c.ny;
    const size_t fcells = s->frame ? (size_t)frame_cells(c.nx, c.ny, s->g) : 0;
    h.state_bytes = sizeof(double) * s->nv * cells;
    h.frame_bytes = sizeof(double) * s->nv * fcells;
    std::vector<double> host(s->nv * cells + s->nv * fcells);
    const double* src = s->buf[d.cur & 1];
    for (int k = 0; k < s->nv; ++k)
        CUDA_TRY(cudaMemcpy2DAsync(host.data() + k * cells, c.nx * sizeof(double),
                                   src + k * s->plane, s->pitch * sizeof(double),
                                   c.nx * sizeof(double), c.ny, cudaMemcpyDeviceToHost, s->stream));
    if (s->frame)
        CUDA_TRY(cudaMemcpyAsync(host.data() + s->nv * cells, s->frame, h.frame_bytes,
                                 cudaMemcpyDeviceToHost, s->stream));
    CUDA_TRY(cudaStreamSynchronize(s->stream));
    FILE* f = fopen(path, "wb");
    if (!f) return fail(CFD_ERR_INVALID, "cannot write %s", path);
    bool ok = fwrite(&h, sizeof h, 1, f) == 1 &&
              fwrite(host.data(), sizeof(double), host.size(), f) == host.size();
    ok = (fclose(f) == 0) && ok;
    return ok ? CFD_OK : fail(CFD_ERR_INVALID, "short write to %s", path);
}

int cfd_checkpoint_load(cfd_solver* s, const char* path) {
    if (!s || !path) return fail(CFD_ERR_INVALID, "null argument");
    const cfd_config& c = s->cfg;
    FILE* f = fopen(path, "rb");
    if (!f) return fail(CFD_ERR_INVALID, "cannot open %s", path);
    CkptHeader h;
    int r = ckpt_read_header(f, h);
    if (r) {
        fclose(f);
        return fail(r, "%s is not a checkpoint", path);
    }
    if (h.cfg.precision != CFD_PREC_FP64 || h.cfg.model != c.model || h.cfg.nx != c.nx ||
        h.cfg.ny != c.ny || h.g != s->g || h.cfg.dx != c.dx || h.cfg.dy != c.dy) {
        fclose(f);
        return fail(CFD_ERR_INVALID, "checkpoint %s holds a different solve", path);
    }
    const size_t cells = (size_t)c.nx * c.ny;
    const size_t fcells = (size_t)frame_cells(c.nx, c.ny, s->g);
    if (h.state_bytes != sizeof(double) * s->nv * cells ||
        (h.has_frame && h.frame_bytes != sizeof(double) * s->nv * fcells)) {
        fclose(f);
        return fail(CFD_ERR_INVALID, "checkpoint %s has inconsistent sizes", path);
    }
    std::vector<double> host(s->nv * cells + (h.has_frame ? s->nv * fcells : 0));
    bool ok = fread(host.data(), sizeof(double), host.size(), f) == host.size();
    fclose(f);
    if (!ok) return fail(CFD_ERR_INVALID, "checkpoint %s is truncated", path);
    for (int k = 0; k < s->nv; ++k)
        CUDA_TRY(cudaMemcpy2DAsync(s->buf[0] + k * s->plane, s->pitch * sizeof(double),
                                   host.data() + k * cells, c.nx * sizeof(double),
                                   c.nx * sizeof(double), c.ny, cudaMemcpyHostToDevice, s->stream));
    DevState d;
    memset(&d, 0, sizeof d);
    d.t = h.t;
    d.dt = h.dt;
    d.T = c.T;
    d.cfl = c.cfl;
    d.maxu = h.maxu;
    d.maxv = h.maxv;
    d.mass1 = h.mass1;
    d.mass2 = h.mass2;
    d.dx = c.dx;
    d.dy = c.dy;
    d.n = h.n;
    d.done = h.t >= c.T;
    CUDA_TRY(cudaMemcpyAsync(s->dst, &d, sizeof d, cudaMemcpyHostToDevice, s->stream));
    CUDA_TRY(cudaMemcpyAsync(s->counters, h.counters, sizeof h.counters, cudaMemcpyHostToDevice,
                             s->stream));
    if (s->frame) {
        if (h.has_frame)
            CUDA_TRY(cudaMemcpyAsync(s->frame, host.data() + s->nv * cells,
                                     sizeof(double) * s->nv * fcells, cudaMemcpyHostToDevice,
                                     s->stream));
        else if ((r = frame_from_state(s)))
            return r;
    }
    // the host vectors are pageable: the copies have read them when the calls return
    CUDA_TRY(cudaStreamSynchronize(s->stream));
    s->uploaded = true;
    return CFD_OK;
}

int cfd_set_reference_ghosts(cfd_solver* s, int enable) {
    if (!s) return fail(CFD_ERR_INVALID, "null solver");
    const cfd_config& c = s->cfg;
    if (s->graph) {  // the captured steps change
        CUDA_TRY(cudaStreamSynchronize(s->stream));
        cudaGraphExecDestroy(s->graph);
        s->graph = nullptr;
    }
    if (!enable) {
        if (s->frame) {
            CUDA_TRY(cudaStreamSynchronize(s->stream));
            cudaFree(s->frame);
            s->frame = nullptr;
        }
        s->ref_ghosts = false;
        return CFD_OK;
    }
    if (!s->frame) {
        size_t bytes = sizeof(double) * s->nv * frame_cells(c.nx, c.ny, s->g);
        cudaError_t e = cudaMalloc(&s->frame, bytes);
        if (e != cudaSuccess) {
            s->frame = nullptr;
            return fail(CFD_ERR_NOMEM, "ghost frame: %s", cudaGetErrorString(e));
        }
        CUDA_TRY(cudaMemsetAsync(s->frame, 0, bytes, s->stream));
        int r;
        if (s->uploaded && (r = enqueue_frame_snapshot(s, 0, true))) return r;
    }
    s->ref_ghosts = true;
    return CFD_OK;
}

int cfd_set_kernel_timing(cfd_solver* s, int enable) {
    if (!s) return fail(CFD_ERR_INVALID, "null solver");
    s->timing = enable != 0;
    return CFD_OK;
}

int cfd_kernel_times(cfd_solver* s, double* ms, int* launches) {
    if (!s || !ms || !launches) return fail(CFD_ERR_INVALID, "null argument");
    CUDA_TRY(cudaStreamSynchronize(s->stream));
    for (int d = 0; d < 2; ++d) {
        for (auto& pr : s->ev[d]) {
            float m = 0.f;
            CUDA_TRY(cudaEventElapsedTime(&m, pr.first, pr.second));
            s->ev_ms[d] += m;
            s->ev_n[d] += 1;
            cudaEventDestroy(pr.first);
            cudaEventDestroy(pr.second);
        }
        s->ev[d].clear();
        ms[d] = s->ev_ms[d];
        launches[d] = s->ev_n[d];
    }
    return CFD_OK;
}

int cfd_reset_kernel_times(cfd_solver* s) {
    if (!s) return fail(CFD_ERR_INVALID, "null solver");
    double ms[2];
    int n[2];
    int r = cfd_kernel_times(s, ms, n);
    s->ev_ms[0] = s->ev_ms[1] = 0.0;
    s->ev_n[0] = s->ev_n[1] = 0;
    return r;
}

int cfd_reset_counters(cfd_solver* s) {
    if (!s) return fail(CFD_ERR_INVALID, "null solver");
    CUDA_TRY(cudaMemsetAsync(s->counters, 0, CNT_N * sizeof(unsigned long long), s->stream));
    return CFD_OK;
}

int cfd_synchronize(cfd_solver* s) {
    if (!s) return fail(CFD_ERR_INVALID, "null solver");
    CUDA_TRY(cudaStreamSynchronize(s->stream));
    return CFD_OK;
}

int cfd_state_device(cfd_solver* s, const void** dev_ptr, int64_t* plane, int* pitch) {
    if (!s || !dev_ptr) return fail(CFD_ERR_INVALID, "null argument");
    int cur, r;
    if ((r = current_buffer(s, cur))) return r;
    *dev_ptr = s->buf[cur];
    if (plane) *plane = s->plane;
    if (pitch) *pitch = s->pitch;
    return CFD_OK;
}

int cfd_face_flux(const cfd_config* cfg, int nfaces, const double* stencils, double dt, double dx,
                  double* flux, double* u_star, double* z_star) {
    cfd_config c = *cfg;
    if (c.nx < 2) c.nx = 2;
    if (c.ny < 2) c.ny = 2;
    if (c.dx <= 0) c.dx = 1;
    if (c.dy <= 0) c.dy = 1;
    if (c.cfl <= 0) c.cfl = 0.5;
    c.precision = CFD_PREC_FP64;
    int r = validate_config(&c);
    if (r) return r;
    if (nfaces <= 0) return CFD_OK;
    int nv = cfd_nvar(c.model);
    int m = c.flux_solver == CFD_FLUX_GODUNOV ? 2 : 4;
    size_t in_b = sizeof(double) * (size_t)nfaces * m * nv;
    size_t fl_b = sizeof(double) * (size_t)nfaces * nv;
    double *d_in = nullptr, *d_fl = nullptr, *d_us = nullptr, *d_zs = nullptr;
    cudaError_t e = cudaMalloc(&d_in, in_b);
    if (e == cudaSuccess) e = cudaMalloc(&d_fl, fl_b);
    if (e == cudaSuccess) e = cudaMalloc(&d_us, sizeof(double) * nfaces);
    if (e == cudaSuccess) e = cudaMalloc(&d_zs, sizeof(double) * nfaces);
    if (e == cudaSuccess) e = cudaMemcpy(d_in, stencils, in_b, cudaMemcpyHostToDevice);
    if (e == cudaSuccess) {
        Eos q = make_eos(c);
        double s_half = 0.5 * (dt / dx);
        int blocks = (nfaces + 127) / 128;
        if (c.model == CFD_MODEL_EULER)
            face_flux_kernel<MODEL_EULER><<<blocks, 128>>>(nfaces, d_in, q, c.limiter, c.wavespeed,
                                                          c.flux_solver == CFD_FLUX_GODUNOV,
                                                          c.z_min, s_half, d_fl, d_us, nullptr);
        else
            face_flux_kernel<MODEL_ALLAIRE><<<blocks, 128>>>(
                nfaces, d_in, q, c.limiter, c.wavespeed, c.flux_solver == CFD_FLUX_GODUNOV,
                c.z_min, s_half, d_fl, d_us, d_zs);
        e = cudaGetLastError();
    }
    if (e == cudaSuccess) e = cudaMemcpy(flux, d_fl, fl_b, cudaMemcpyDeviceToHost);
    if (e == cudaSuccess && u_star)
        e = cudaMemcpy(u_star, d_us, sizeof(double) * nfaces, cudaMemcpyDeviceToHost);
    if (e == cudaSuccess && z_star && c.model == CFD_MODEL_ALLAIRE)
        e = cudaMemcpy(z_star, d_zs, sizeof(double) * nfaces, cudaMemcpyDeviceToHost);
    cudaFree(d_in);
    cudaFree(d_fl);
    cudaFree(d_us);
    cudaFree(d_zs);
    if (e != cudaSuccess) return fail(CFD_ERR_CUDA, "face flux: %s", cudaGetErrorString(e));
    return CFD_OK;
}

}  // extern "C"
