// Batched solves: many independent grids of uneven sizes advanced together.
//
// A batch owns device state for each member solve (instance) and advances
// all active instances by one split step per "tick": one persistent x-sweep
// launch and one persistent y-sweep launch per model present, over a tile
// list that covers every active instance (x: warp segments, csrc/cfd_march.cuh;
// y: shared-memory tiles, csrc/cfd_mixed.cuh, or marching strips).  Each instance
// keeps its own time-loop state (n, t, dt, T, max_steps), picks its own dt
// after each step and stops on its own.  Ticks are captured into a CUDA graph
// that is replayed until the membership changes.  Instances are admitted
// against a device-memory budget, so a server can keep adding work while
// others run.
//
// Precision, per member: the mixed form (FP32 + compensation word state;
// cfd_mixed.cuh) or the fast FP64 form (cfd_fast64.cuh), which stores FP64
// values in the same planes; each (model, form) pair has its own tile lists
// and launches.  The bit-identical FP64 form uses cfd_solver (cfd_api.cu).
#include <cuda_runtime.h>

#include <algorithm>
#include <cmath>
#include <cstdint>
#include <cstring>
#include <map>
#include <new>
#include <string>
#include <utility>
#include <vector>

#include "../../include/cfdgpu.h"
#include "cfd_checkpoint.h"
#include "cfd_error.h"
#include "cfd_fast64.cuh"
#include "cfd_ic.h"
#include "cfd_march.cuh"
#include "cfd_mixed.cuh"
#include "cfd_pool.h"
#include "ic_builders.h"

using namespace cfd;
using namespace cfd::mixed;

namespace {

#define BTRY(expr)                                                                          \
    do {                                                                                    \
        cudaError_t e_ = (expr);                                                            \
        if (e_ != cudaSuccess)                                                              \
            return cfd_fail(e_ == cudaErrorMemoryAllocation ? CFD_ERR_NOMEM : CFD_ERR_CUDA, \
                            "%s: %s", #expr, cudaGetErrorString(e_));                       \
    } while (0)

// Tile-shape variants the autotuner chooses from: (TS along, NA across),
// each keeping every phase of a 256-thread CTA a single pass.
struct Shape {
    int ts, na;
};
// x: warp segments of kSegCells columns (cfd_march.cuh), the only x form (it
// measured 13-25 % faster than every tile shape, and a single x form keeps
// results independent of the autotuner's choice); their row count is chosen
// per launch (seg_rows), kSegRows is the nominal one.
// y: three tile shapes, and shape 3 = marching strips of 32 columns
// (cfd_march.cuh), bit-identical to the tiles; their length is chosen per
// launch (march_rows), kMarchMaxRows is the nominal one.
constexpr Shape kShapesX[] = {{kSegCells, kSegRows}};
constexpr Shape kShapesY[] = {{28, 8}, {60, 4}, {12, 16}, {kMarchMaxRows, 32}};
constexpr int kNumShapesX = 1, kNumShapesY = 4;
constexpr int kMarchShape = 3;

// Persistent launch: as many CTAs as fit on the device at once (occupancy
// of this variant), never more than there are tiles.
template <int MODEL, int DIR, int TS, int NA>
int launch_t(const MixedArgs& a, int sms, cudaStream_t st) {
    constexpr int smem = MTile<MODEL, DIR, TS, NA>::SMEM;
    static int per_sm = 0;
    if (!per_sm) {
        cudaError_t e = cudaFuncSetAttribute(mixed_sweep_kernel<MODEL, DIR, TS, NA>,
                                             cudaFuncAttributeMaxDynamicSharedMemorySize, smem);
        if (e != cudaSuccess) return cfd_fail(CFD_ERR_CUDA, "smem attribute: %s", cudaGetErrorString(e));
        e = cudaOccupancyMaxActiveBlocksPerMultiprocessor(
            &per_sm, mixed_sweep_kernel<MODEL, DIR, TS, NA>, 256, smem);
        if (e != cudaSuccess || per_sm < 1) per_sm = 1;
    }
    int grid = std::max(1, std::min(a.ntiles, per_sm * sms));
    MixedArgs b = a;
    b.chunk = (a.ntiles + grid - 1) / grid;
    grid = (a.ntiles + b.chunk - 1) / b.chunk;
    mixed_sweep_kernel<MODEL, DIR, TS, NA><<<grid, 256, smem, st>>>(b);
    cudaError_t e = cudaGetLastError();
    if (e != cudaSuccess) return cfd_fail(CFD_ERR_CUDA, "mixed sweep launch: %s", cudaGetErrorString(e));
    return CFD_OK;
}

// Resident 4-warp CTAs per SM of the marching sweep.
template <int MODEL, int DIR>
int march_per_sm() {
    static int per_sm = 0;
    if (!per_sm) {
        cudaError_t e = cudaOccupancyMaxActiveBlocksPerMultiprocessor(
            &per_sm, mixed_march_kernel<MODEL, DIR>, 128, march_smem_bytes<MODEL>());
        if (e != cudaSuccess || per_sm < 1) per_sm = 1;
    }
    return per_sm;
}

// Persistent marching y sweep (4-warp CTAs): as many warps as fit on the
// device (never more than there are strips), each walking every W-th strip.
template <int MODEL, int DIR>
int launch_march(const MixedArgs& a, int sms, cudaStream_t st) {
    const int warps = std::max(1, std::min(a.ntiles, march_per_sm<MODEL, DIR>() * sms * 4));
    mixed_march_kernel<MODEL, DIR><<<(warps + 3) / 4, 128, march_smem_bytes<MODEL>(), st>>>(a);
    cudaError_t e = cudaGetLastError();
    if (e != cudaSuccess) return cfd_fail(CFD_ERR_CUDA, "march launch: %s", cudaGetErrorString(e));
    return CFD_OK;
}

// Persistent warp-segment x sweep (4-warp CTAs), launched like the marching one.
template <int MODEL>
int segment_per_sm() {
    static int per_sm = 0;
    if (!per_sm) {
        cudaError_t e = cudaOccupancyMaxActiveBlocksPerMultiprocessor(
            &per_sm, mixed_segment_x_kernel<MODEL>, 128, seg_smem_bytes<MODEL>());
        if (e != cudaSuccess || per_sm < 1) per_sm = 1;
    }
    return per_sm;
}

template <int MODEL>
int launch_segment(const MixedArgs& a, int sms, cudaStream_t st) {
    const int warps = std::max(1, std::min(a.ntiles, segment_per_sm<MODEL>() * sms * 4));
    mixed_segment_x_kernel<MODEL><<<(warps + 3) / 4, 128, seg_smem_bytes<MODEL>(), st>>>(a);
    cudaError_t e = cudaGetLastError();
    if (e != cudaSuccess) return cfd_fail(CFD_ERR_CUDA, "segment launch: %s", cudaGetErrorString(e));
    return CFD_OK;
}

// The fast FP64 form's sweeps (cfd_fast64.cuh), launched like the mixed
// warp forms: x by warp segments, y by marching strips.
template <int MODEL>
int march64_per_sm() {
    static int per_sm = 0;
    if (!per_sm) {
        cudaError_t e = cudaOccupancyMaxActiveBlocksPerMultiprocessor(
            &per_sm, fast::fast_march_kernel<MODEL>, 128, fast::march64_smem_bytes<MODEL>());
        if (e != cudaSuccess || per_sm < 1) per_sm = 1;
    }
    return per_sm;
}

template <int MODEL>
int segment64_per_sm() {
    static int per_sm = 0;
    if (!per_sm) {
        cudaError_t e = cudaOccupancyMaxActiveBlocksPerMultiprocessor(
            &per_sm, fast::fast_segment_x_kernel<MODEL>, 128, fast::segment64_smem_bytes<MODEL>());
        if (e != cudaSuccess || per_sm < 1) per_sm = 1;
    }
    return per_sm;
}

template <int MODEL>
int launch_fast(int dir, const MixedArgs& a, int sms, cudaStream_t st) {
    const int per_sm = dir == DIR_X ? segment64_per_sm<MODEL>() : march64_per_sm<MODEL>();
    const int warps = std::max(1, std::min(a.ntiles, per_sm * sms * 4));
    if (dir == DIR_X)
        fast::fast_segment_x_kernel<MODEL><<<(warps + 3) / 4, 128, fast::segment64_smem_bytes<MODEL>(), st>>>(a);
    else
        fast::fast_march_kernel<MODEL><<<(warps + 3) / 4, 128, fast::march64_smem_bytes<MODEL>(), st>>>(a);
    cudaError_t e = cudaGetLastError();
    if (e != cudaSuccess) return cfd_fail(CFD_ERR_CUDA, "fast FP64 sweep launch: %s", cudaGetErrorString(e));
    return CFD_OK;
}

template <int MODEL>
int launch_shape(int dir, int shape, const MixedArgs& a, int grid, cudaStream_t st) {
    if (dir == DIR_X) return launch_segment<MODEL>(a, grid, st);
    switch (shape) {
        case 0: return launch_t<MODEL, DIR_Y, 28, 8>(a, grid, st);
        case 1: return launch_t<MODEL, DIR_Y, 60, 4>(a, grid, st);
        case kMarchShape: return launch_march<MODEL, DIR_Y>(a, grid, st);
        default: return launch_t<MODEL, DIR_Y, 12, 16>(a, grid, st);
    }
}

int tiles_for(int nx, int ny, int dir, Shape s) {
    int len = dir == DIR_X ? nx : ny, wid = dir == DIR_X ? ny : nx;
    return ((len + s.ts - 1) / s.ts) * ((wid + s.na - 1) / s.na);
}

// Strip length of a marching launch over strips of 32 columns of the given
// grids: a warp walks ceil(strips / slots) strips one after the other, each
// costing its length plus the 4 halo rows, so the length with the fewest
// (rounds x (rows + 4)) is taken, the longest on ties.  Grids with few
// strips get shorter ones, so that they still fill the resident warps.
int march_rows(const std::vector<std::pair<int, int>>& grids, long long slots) {
    int best = kMarchMaxRows;
    long long best_cost = -1;
    for (int rows = kMarchMaxRows; rows >= kMarchMinRows; rows -= 4) {
        long long strips = 0;
        for (const auto& g : grids) strips += (long long)((g.first + 31) / 32) * ((g.second + rows - 1) / rows);
        if (!strips) return kMarchMaxRows;
        const long long cost = (strips + slots - 1) / slots * (rows + 4);
        if (best_cost < 0 || cost < best_cost) {
            best_cost = cost;
            best = rows;
        }
    }
    return best;
}

// Row count of the x sweep's warp segments over the given grids: tiles of
// kSegCells columns, a warp walks ceil(tiles / slots) of them one after the
// other, each costing its rows plus about two rows' worth of setup (the
// member's constants, the first row's load), so the count with the fewest
// (rounds x (rows + 2)) is taken, the largest on ties.  A lone grid that
// leaves resident warps idle at 32 rows gets shorter tiles.
int seg_rows(const std::vector<std::pair<int, int>>& grids, long long slots) {
    int best = kSegRows;
    long long best_cost = -1;
    for (int rows = kSegRows; rows >= kSegMinRows; rows -= 2) {
        long long tiles = 0;
        for (const auto& g : grids)
            tiles += (long long)((g.first + kSegCells - 1) / kSegCells) * ((g.second + rows - 1) / rows);
        if (!tiles) return kSegRows;
        const long long cost = (tiles + slots - 1) / slots * (rows + 2);
        if (best_cost < 0 || cost < best_cost) {
            best_cost = cost;
            best = rows;
        }
    }
    return best;
}

// ---- conversion kernels ----------------------------------------------------

// One cell of an FP64 member's packed planes (the storage of cfd_fast64.cuh).
__device__ __forceinline__ void store_packed64(const Inst& I, int buf, long long o, const double* U) {
    reinterpret_cast<double2*>(I.q4[buf][0])[o] = make_double2(U[0], U[1]);
    reinterpret_cast<double2*>(I.q4[buf][1])[o] = make_double2(U[2], U[3]);
    if (I.nv == 6) {
        reinterpret_cast<double*>(I.q2[buf][0])[o] = U[4];
        reinterpret_cast<double*>(I.q2[buf][1])[o] = U[5];
    }
}
__device__ __forceinline__ void load_packed64(const Inst& I, int buf, long long o, double* U) {
    const double2 a = reinterpret_cast<const double2*>(I.q4[buf][0])[o];
    const double2 b = reinterpret_cast<const double2*>(I.q4[buf][1])[o];
    U[0] = a.x;
    U[1] = a.y;
    U[2] = b.x;
    U[3] = b.y;
    if (I.nv == 6) {
        U[4] = reinterpret_cast<const double*>(I.q2[buf][0])[o];
        U[5] = reinterpret_cast<const double*>(I.q2[buf][1])[o];
    }
}

// Ghosted FP64 AoS grid -> packed planes (value/compensation, or FP64), plus
// an FP64 SoA copy for the initial wave-speed reduction.
__global__ void ghosted_to_mixed(const double* __restrict__ src, Inst I,
                                 double* __restrict__ soa, int g) {
    long long n = (long long)I.nx * I.ny;
    const int nv = I.nv;
    for (long long idx = blockIdx.x * (long long)blockDim.x + threadIdx.x; idx < n;
         idx += (long long)gridDim.x * blockDim.x) {
        int i = (int)(idx / I.nx), j = (int)(idx % I.nx);
        const double* c = src + ((long long)(i + g) * (I.nx + 2 * g) + (j + g)) * nv;
        long long o = (long long)i * I.pitch + j;
        if (I.fp64) {
            double U[6] = {0.0, 0.0, 0.0, 0.0, 0.0, 0.0};
            for (int k = 0; k < nv; ++k) soa[k * I.plane + o] = U[k] = c[k];
            store_packed64(I, 0, o, U);
            continue;
        }
        float h[6], l[6];
        for (int k = 0; k < nv; ++k) {
            double x = c[k];
            h[k] = (float)x;
            l[k] = (float)(x - (double)h[k]);
            soa[k * I.plane + o] = x;
        }
        I.q4[0][0][o] = make_float4(h[0], h[1], h[2], h[3]);
        I.q4[0][1][o] = make_float4(l[0], l[1], l[2], l[3]);
        if (nv == 6) {
            I.q2[0][0][o] = make_float2(h[4], h[5]);
            I.q2[0][1][o] = make_float2(l[4], l[5]);
        }
    }
}

// FP64 SoA planes (the instance's pitch and plane) -> packed planes of
// buffer 0.
__global__ void soa_to_mixed(const double* __restrict__ soa, Inst I) {
    long long n = (long long)I.nx * I.ny;
    const int nv = I.nv;
    for (long long idx = blockIdx.x * (long long)blockDim.x + threadIdx.x; idx < n;
         idx += (long long)gridDim.x * blockDim.x) {
        int i = (int)(idx / I.nx), j = (int)(idx % I.nx);
        long long o = (long long)i * I.pitch + j;
        if (I.fp64) {
            double U[6] = {0.0, 0.0, 0.0, 0.0, 0.0, 0.0};
            for (int k = 0; k < nv; ++k) U[k] = soa[k * I.plane + o];
            store_packed64(I, 0, o, U);
            continue;
        }
        float h[6], l[6];
        for (int k = 0; k < nv; ++k) {
            double x = soa[k * I.plane + o];
            h[k] = (float)x;
            l[k] = (float)(x - (double)h[k]);
        }
        I.q4[0][0][o] = make_float4(h[0], h[1], h[2], h[3]);
        I.q4[0][1][o] = make_float4(l[0], l[1], l[2], l[3]);
        if (nv == 6) {
            I.q2[0][0][o] = make_float2(h[4], h[5]);
            I.q2[0][1][o] = make_float2(l[4], l[5]);
        }
    }
}

// Packed planes of buffer `buf` (< 0: the current one) -> FP64 AoS with the
// boundary mirror in the ghost strips (g = 0: interior only); corners are zero.
// Mixed members give value + compensation, FP64 members their values.
__global__ void mixed_to_ghosted(Inst I, int buf, double* __restrict__ dst, int g, int im,
                                 int it, int use_bc) {
    if (buf < 0) buf = I.st->cur & 1;  // the current buffer
    const int nx = I.nx, ny = I.ny, nv = I.nv;
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
        if (j < 0) { sj = -j - 1; if (use_bc && I.bc[0]) neg = im; }
        else if (j >= nx) { sj = 2 * nx - 1 - j; if (use_bc && I.bc[1]) neg = im; }
        if (i < 0) { si = -i - 1; if (use_bc && I.bc[2]) neg = it; }
        else if (i >= ny) { si = 2 * ny - 1 - i; if (use_bc && I.bc[3]) neg = it; }
        long long o = (long long)si * I.pitch + sj;
        double v[6] = {0.0, 0.0, 0.0, 0.0, 0.0, 0.0};
        if (I.fp64) {
            load_packed64(I, buf, o, v);
        } else {
            float4 a = I.q4[buf][0][o], b = I.q4[buf][1][o];
            v[0] = (double)a.x + b.x;
            v[1] = (double)a.y + b.y;
            v[2] = (double)a.z + b.z;
            v[3] = (double)a.w + b.w;
            if (nv == 6) {
                float2 c = I.q2[buf][0][o], e = I.q2[buf][1][o];
                v[4] = (double)c.x + e.x;
                v[5] = (double)c.y + e.y;
            }
        }
        for (int k = 0; k < nv; ++k) d[k] = (k == neg) ? -v[k] : v[k];
    }
}

template <int MODEL>
__global__ void init_reduce(const double* __restrict__ in, long long plane, int pitch, int nx,
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
        is_last = atomicAdd(&st->ticket, 1u) == gridDim.x - 1;
    }
    __syncthreads();
    if (is_last) {
        __threadfence();
        finish_reduction(st, partials, gridDim.x, 0, 0.0, 0);
    }
}

constexpr int kInitBlocks = 148 * 2;

struct PollRec {
    double t;
    int n, done;
};

// Time state of every member into one array (one copy to the host).
__global__ void gather_status(const Inst* __restrict__ insts, int n, PollRec* __restrict__ out) {
    int i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= n) return;
    const DevState* st = insts[i].st;
    out[i].t = st->t;
    out[i].n = st->n;
    out[i].done = st->done || st->n >= insts[i].max_steps;
}

// A status gather of every member queued on the batch stream and copied to
// pinned memory; read once its event has completed.
struct Gather {
    PollRec* d = nullptr;
    PollRec* h = nullptr;  // pinned
    int cap = 0;
    cudaEvent_t ev = nullptr;
    bool pending = false;
    std::vector<int> ids;  // member ids of the gathered entries
};

struct Member {
    bool final = false;   // seen done: later sweeps leave its state alone
    int id;
    cfd_config cfg;
    Inst inst;          // host copy of the device descriptor
    void* mem = nullptr;  // one allocation: buffers, state, partials
    size_t bytes = 0;
    int max_steps;
};

}  // namespace

struct cfd_batch {
    cudaStream_t stream = nullptr;
    bool own_stream = false;
    size_t budget = 0, used = 0;
    int next_id = 1;
    std::vector<Member> members;
    Inst* d_insts = nullptr;
    int d_insts_cap = 0;
    // tile lists per (model, dir): device arrays
    TileEnt* d_tiles = nullptr;
    size_t d_tiles_cap = 0;
    struct Group {
        int model, fp64, dir, shape, ntiles, offset;
        int rows;  // marching strips: cells along the sweep per strip
    };
    std::vector<Group> groups;
    bool dirty = true;
    // [model][dir]; y sweeps march by default (measured fastest on B200 for
    // both models, and the strips adapt to the members)
    int shape[2][2] = {{0, kMarchShape}, {0, kMarchShape}};
    int march_fixed[2] = {0, 0};  // strip length set by the caller (0: chosen per tile list)
    int march_used[2] = {0, 0};   // strip length of the current mixed tile list
    int march_used64[2] = {0, 0}; // strip length of the current fast FP64 tile list
    int seg_used[2][2] = {};      // [model][fast FP64] rows of the current x segments
    int sms = 148;
    // graph of `graph_steps` ticks for the current membership
    cudaGraphExec_t graph = nullptr;
    int graph_steps = 0;
    // autotuning state
    bool tuned = false;
    int tune_override = -1;
    // uploads run on their own stream; batch-stream work waits for them
    cudaStream_t copy = nullptr;
    std::vector<cudaEvent_t> pending;
    // status of every member gathered on the device, read with one copy
    PollRec* d_poll = nullptr;
    PollRec* h_poll = nullptr;  // pinned
    int poll_cap = 0;
    // asynchronous status gathers of cfd_batch_step, one per chunk of ticks
    // in flight (finished members leave the tile lists one chunk later)
    Gather async[2];
    int async_next = 0;  // the slot the next chunk's gather uses
    // the caller's two-phase status read (cfd_batch_poll_issue / _collect)
    Gather issued;
};

namespace {

// Orders the batch stream after every upload queued on the copy stream.
int wait_uploads(cfd_batch* b) {
    cudaError_t r = cudaSuccess;
    for (cudaEvent_t e : b->pending) {
        if (r == cudaSuccess) r = cudaStreamWaitEvent(b->stream, e, 0);
        cudaEventDestroy(e);  // its resources go once it has completed
    }
    b->pending.clear();
    return r == cudaSuccess ? CFD_OK
                            : cfd_fail(CFD_ERR_CUDA, "upload wait: %s", cudaGetErrorString(r));
}

int build_tables(cfd_batch* b) {
    if (int r = wait_uploads(b)) return r;
    if (!b->dirty) return CFD_OK;
    b->groups.clear();
    // the x segments' row count and the y shape of each (model, form), with
    // the strip length of a marching sweep; the fast FP64 form always
    // marches in y
    Shape shape_x[2][2], shape_y[2][2];
    for (int model = 0; model < 2; ++model)
        for (int f64 = 0; f64 < 2; ++f64) {
            const int shp = f64 ? kMarchShape : b->shape[model][DIR_Y];
            shape_x[model][f64] = kShapesX[0];
            shape_y[model][f64] = kShapesY[shp];
            int& used = f64 ? b->march_used64[model] : b->march_used[model];
            used = 0;
            b->seg_used[model][f64] = 0;
            std::vector<std::pair<int, int>> grids;
            for (const Member& m : b->members)
                if (m.cfg.model == model && m.inst.fp64 == f64 && !m.final)
                    grids.emplace_back(m.cfg.nx, m.cfg.ny);
            if (grids.empty()) continue;
            const int seg_sm =
                f64 ? (model == CFD_MODEL_EULER ? segment64_per_sm<MODEL_EULER>()
                                                : segment64_per_sm<MODEL_ALLAIRE>())
                    : (model == CFD_MODEL_EULER ? segment_per_sm<MODEL_EULER>()
                                                : segment_per_sm<MODEL_ALLAIRE>());
            shape_x[model][f64].na = seg_rows(grids, (long long)seg_sm * b->sms * 4);
            b->seg_used[model][f64] = shape_x[model][f64].na;
            if (shp != kMarchShape) continue;
            const int per_sm =
                f64 ? (model == CFD_MODEL_EULER ? march64_per_sm<MODEL_EULER>()
                                                : march64_per_sm<MODEL_ALLAIRE>())
                    : (model == CFD_MODEL_EULER ? march_per_sm<MODEL_EULER, DIR_Y>()
                                                : march_per_sm<MODEL_ALLAIRE, DIR_Y>());
            shape_y[model][f64].ts = b->march_fixed[model]
                                         ? b->march_fixed[model]
                                         : march_rows(grids, (long long)per_sm * b->sms * 4);
            used = shape_y[model][f64].ts;
        }
    std::vector<Inst> insts(b->members.size());
    for (size_t i = 0; i < b->members.size(); ++i) {
        Member& m = b->members[i];
        int model = m.cfg.model;
        m.inst.tiles_x = tiles_for(m.cfg.nx, m.cfg.ny, DIR_X, shape_x[model][m.inst.fp64]);
        m.inst.tiles_y = tiles_for(m.cfg.nx, m.cfg.ny, DIR_Y, shape_y[model][m.inst.fp64]);
        insts[i] = m.inst;
    }
    // largest instances first within each group so the tail of a sweep is
    // made of small tiles of small solves
    std::vector<int> order(b->members.size());
    for (size_t i = 0; i < order.size(); ++i) order[i] = (int)i;
    std::sort(order.begin(), order.end(), [&](int x, int y) {
        return (long long)b->members[x].cfg.nx * b->members[x].cfg.ny >
               (long long)b->members[y].cfg.nx * b->members[y].cfg.ny;
    });
    std::vector<TileEnt> all;
    for (int model = 0; model < 2; ++model)
        for (int f64 = 0; f64 < 2; ++f64)
            for (int dir = 0; dir < 2; ++dir) {
                cfd_batch::Group g;
                g.model = model;
                g.fp64 = f64;
                g.dir = dir;
                g.shape = f64 ? (dir == DIR_X ? 0 : kMarchShape) : b->shape[model][dir];
                g.offset = (int)all.size();
                const Shape sh = dir == DIR_X ? shape_x[model][f64] : shape_y[model][f64];
                g.rows = dir == DIR_X ? sh.na : sh.ts;
                for (int idx : order) {
                    const Member& m = b->members[idx];
                    // finished members have no tiles
                    if (m.cfg.model != model || m.inst.fp64 != f64 || m.final) continue;
                    const int len = dir == DIR_X ? m.cfg.nx : m.cfg.ny;
                    const int wid = dir == DIR_X ? m.cfg.ny : m.cfg.nx;
                    const int along = (len + sh.ts - 1) / sh.ts;
                    const int nt = dir == DIR_X ? insts[idx].tiles_x : insts[idx].tiles_y;
                    for (int t = 0; t < nt; ++t) {
                        TileEnt e;
                        e.inst = idx;
                        e.local = t;
                        e.a_org = (t % along) * sh.ts - 2;
                        e.b_org = (t / along) * sh.na;
                        e.len = len;
                        e.wid = wid;
                        e.max_steps = insts[idx].max_steps;
                        e.active = insts[idx].active;
                        all.push_back(e);
                    }
                }
                g.ntiles = (int)all.size() - g.offset;
                if (g.ntiles) b->groups.push_back(g);
            }
    if ((int)insts.size() > b->d_insts_cap) {
        pool_free(b->d_insts, b->stream);
        b->d_insts = nullptr;
        int cap = std::max<int>(16, (int)insts.size() * 2);
        BTRY(pool_alloc(reinterpret_cast<void**>(&b->d_insts), sizeof(Inst) * cap, b->stream));
        b->d_insts_cap = cap;
    }
    if (all.size() > b->d_tiles_cap) {
        pool_free(b->d_tiles, b->stream);
        b->d_tiles = nullptr;
        size_t cap = std::max<size_t>(1024, all.size() * 2);
        BTRY(pool_alloc(reinterpret_cast<void**>(&b->d_tiles), sizeof(TileEnt) * cap, b->stream));
        b->d_tiles_cap = cap;
    }
    if (!insts.empty())
        BTRY(cudaMemcpyAsync(b->d_insts, insts.data(), sizeof(Inst) * insts.size(),
                             cudaMemcpyHostToDevice, b->stream));
    if (!all.empty())
        BTRY(cudaMemcpyAsync(b->d_tiles, all.data(), sizeof(TileEnt) * all.size(),
                             cudaMemcpyHostToDevice, b->stream));
    // pageable sources: the host vectors have been read when the copy calls return
    if (b->graph) {
        cudaGraphExecDestroy(b->graph);
        b->graph = nullptr;
    }
    b->dirty = false;
    return CFD_OK;
}

struct Timed {
    int group;
    cudaEvent_t e0, e1;
};

int enqueue_tick(cfd_batch* b, std::vector<Timed>* timing) {
    for (int dir = 0; dir < 2; ++dir)
        for (int gi = 0; gi < (int)b->groups.size(); ++gi) {
            const auto& g = b->groups[gi];
            if (g.dir != dir) continue;
            MixedArgs a;
            a.insts = b->d_insts;
            a.tiles = b->d_tiles + g.offset;
            a.ntiles = g.ntiles;
            a.rows = g.rows;
            cudaEvent_t e0 = nullptr, e1 = nullptr;
            if (timing) {
                cudaEventCreate(&e0);
                cudaEventCreate(&e1);
                cudaEventRecord(e0, b->stream);
            }
            int grid = b->sms;
            int r;
            if (g.fp64)
                r = g.model == CFD_MODEL_EULER ? launch_fast<MODEL_EULER>(dir, a, grid, b->stream)
                                               : launch_fast<MODEL_ALLAIRE>(dir, a, grid, b->stream);
            else
                r = g.model == CFD_MODEL_EULER
                        ? launch_shape<MODEL_EULER>(dir, g.shape, a, grid, b->stream)
                        : launch_shape<MODEL_ALLAIRE>(dir, g.shape, a, grid, b->stream);
            if (timing) {
                cudaEventRecord(e1, b->stream);
                timing->push_back({gi, e0, e1});
            }
            if (r) return r;
        }
    return CFD_OK;
}

size_t member_bytes(const cfd_config& c, size_t* plane_out, int* pitch_out) {
    int nv = cfd_nvar(c.model);
    int pitch = (c.nx + 31) / 32 * 32;
    size_t plane = (size_t)pitch * c.ny;
    int ty = 0;
    for (int s = 0; s < kNumShapesX; ++s) ty = std::max(ty, tiles_for(c.nx, c.ny, DIR_X, kShapesX[s]));
    for (int s = 0; s < kNumShapesY; ++s) ty = std::max(ty, tiles_for(c.nx, c.ny, DIR_Y, kShapesY[s]));
    ty = std::max(ty, tiles_for(c.nx, c.ny, DIR_Y, Shape{kMarchMinRows, 32}));  // shortest strips
    int npart = std::max(ty, kInitBlocks);
    size_t bytes = 4 * sizeof(float) * nv * plane  // value/compensation x 2 buffers
                   + 256 + sizeof(DevState) + 4 * sizeof(double) * npart + 4096;
    if (plane_out) *plane_out = plane;
    if (pitch_out) *pitch_out = pitch;
    return bytes;
}

}  // namespace

extern "C" {

int cfd_batch_create(void* stream, size_t device_budget_bytes, cfd_batch** out) {
    if (!out) return cfd_fail(CFD_ERR_INVALID, "null output pointer");
    *out = nullptr;
    int ndev = 0;
    if (cudaGetDeviceCount(&ndev) != cudaSuccess || ndev == 0)
        return cfd_fail(CFD_ERR_CUDA, "no CUDA device available");
    cfd_batch* b = new (std::nothrow) cfd_batch();
    if (!b) return cfd_fail(CFD_ERR_NOMEM, "host allocation failed");
    if (stream) {
        b->stream = (cudaStream_t)stream;
    } else {
        cudaError_t e = cudaStreamCreateWithFlags(&b->stream, cudaStreamNonBlocking);
        if (e != cudaSuccess) {
            delete b;
            return cfd_fail(CFD_ERR_CUDA, "stream: %s", cudaGetErrorString(e));
        }
        b->own_stream = true;
    }
    if (cudaStreamCreateWithFlags(&b->copy, cudaStreamNonBlocking) != cudaSuccess) {
        if (b->own_stream) cudaStreamDestroy(b->stream);
        delete b;
        return cfd_fail(CFD_ERR_CUDA, "copy stream creation failed");
    }
    int dev = 0;
    cudaGetDevice(&dev);
    cudaDeviceGetAttribute(&b->sms, cudaDevAttrMultiProcessorCount, dev);
    if (device_budget_bytes == 0) {
        size_t fr = 0, tot = 0;
        cudaMemGetInfo(&fr, &tot);
        device_budget_bytes = (size_t)(0.8 * (double)fr);
    }
    b->budget = device_budget_bytes;
    *out = b;
    return CFD_OK;
}

int cfd_batch_destroy(cfd_batch* b) {
    if (!b) return CFD_OK;
    cudaStreamSynchronize(b->copy);
    for (cudaEvent_t e : b->pending) cudaEventDestroy(e);
    b->pending.clear();
    cudaStreamSynchronize(b->stream);
    if (b->graph) cudaGraphExecDestroy(b->graph);
    for (auto& m : b->members) pool_free(m.mem, b->stream);
    pool_free(b->d_insts, b->stream);
    pool_free(b->d_tiles, b->stream);
    pool_free(b->d_poll, b->stream);
    for (Gather* g : {&b->async[0], &b->async[1], &b->issued}) pool_free(g->d, b->stream);
    cudaStreamSynchronize(b->stream);
    if (b->h_poll) cudaFreeHost(b->h_poll);
    for (Gather* g : {&b->async[0], &b->async[1], &b->issued}) {
        if (g->h) cudaFreeHost(g->h);
        if (g->ev) cudaEventDestroy(g->ev);
    }
    cudaStreamDestroy(b->copy);
    if (b->own_stream) cudaStreamDestroy(b->stream);
    delete b;
    return CFD_OK;
}

int cfd_batch_member_bytes(const cfd_config* cfg, size_t* bytes) {
    if (!cfg || !bytes) return cfd_fail(CFD_ERR_INVALID, "null argument");
    *bytes = member_bytes(*cfg, nullptr, nullptr);
    return CFD_OK;
}

// Saved state of a member (cfd_batch_restore): its packed planes (nx * ny
// cells each, no padding; value and compensation, or the FP64 form's
// doubles) and its time state.
struct Restore {
    const CkptHeader* h;
    const float4* q4[2];
    const float2* q2[2];
};

// Adds a member whose initial state is either a ghosted AoS host grid or a
// shape program built on the device.  The upload runs on the batch's copy
// stream, so it overlaps sweeps already queued; the next batch operation
// waits for it.

static int add_member(cfd_batch* b, const cfd_config* cfg, const double* host_ic,
                      const std::vector<cfdic::Op>* prog, const cfdic::Eos* prog_eos,
                      int max_steps, int* id_out, const Restore* rs = nullptr) {
    const cfd_config& c = *cfg;
    if (c.model != CFD_MODEL_EULER && c.model != CFD_MODEL_ALLAIRE)
        return cfd_fail(CFD_ERR_INVALID, "unknown model %d", c.model);
    if (c.nx < 2 || c.ny < 2) return cfd_fail(CFD_ERR_INVALID, "grid %dx%d too small", c.nx, c.ny);
    if (c.splitting != CFD_SPLIT_NAIVE)
        return cfd_fail(CFD_ERR_UNSUPPORTED, "batched solves use naive splitting");
    if (!(c.gamma1 > 1.0) || (c.model == CFD_MODEL_ALLAIRE && !(c.gamma2 > 1.0)))
        return cfd_fail(CFD_ERR_INVALID, "gamma must be > 1");
    if (max_steps <= 0) max_steps = 0x7fffffff;
    size_t plane;
    int pitch;
    size_t bytes = member_bytes(c, &plane, &pitch);
    if (b->used + bytes > b->budget)
        return cfd_fail(CFD_ERR_BUDGET, "instance needs %zu bytes, %zu of %zu in use", bytes,
                        b->used, b->budget);
    Member m;
    m.id = b->next_id++;
    m.cfg = c;
    m.max_steps = max_steps;
    m.bytes = bytes;
    BTRY(pool_alloc(&m.mem, bytes, b->copy));
    int nv = cfd_nvar(c.model);
    char* p = static_cast<char*>(m.mem);
    auto take = [&](size_t n) {
        char* q = p;
        p += (n + 255) / 256 * 256;
        return q;
    };
    Inst& I = m.inst;
    memset(&I, 0, sizeof I);
    for (int k = 0; k < 2; ++k)
        for (int w = 0; w < 2; ++w) {
            I.q4[k][w] = reinterpret_cast<float4*>(take(sizeof(float4) * plane));
            I.q2[k][w] = nv == 6 ? reinterpret_cast<float2*>(take(sizeof(float2) * plane)) : nullptr;
        }
    I.st = reinterpret_cast<DevState*>(take(sizeof(DevState)));
    int npart = (int)((bytes - 4 * sizeof(float) * nv * plane - 256 - sizeof(DevState) - 4096) /
                      (4 * sizeof(double)));
    I.partials = reinterpret_cast<double*>(take(4 * sizeof(double) * npart));
    I.plane = (long long)plane;
    I.pitch = pitch;
    I.nx = c.nx;
    I.ny = c.ny;
    I.nv = nv;
    I.model = c.model;
    I.limiter = c.limiter;
    I.wavespeed = c.wavespeed;
    I.godunov = c.flux_solver == CFD_FLUX_GODUNOV;
    I.fix_dy = c.fix_dy_halfstep;
    for (int k = 0; k < 4; ++k) I.bc[k] = c.bc[k];
    I.dx = c.dx;
    I.dy = c.dy;
    I.z_min = c.z_min;
    I.eos.g1 = c.gamma1;
    I.eos.p1 = c.pinf1;
    I.eos.g2 = c.model == CFD_MODEL_ALLAIRE ? c.gamma2 : 1.4;
    I.eos.p2 = c.model == CFD_MODEL_ALLAIRE ? c.pinf2 : 0.0;
    I.eos.gm1_1 = I.eos.g1 - 1.0;
    I.eos.gm1_2 = I.eos.g2 - 1.0;
    I.eos.gp1 = I.eos.g1 * I.eos.p1;
    const double c1 = I.eos.g1 * I.eos.p1 / I.eos.gm1_1, c2 = I.eos.g2 * I.eos.p2 / I.eos.gm1_2;
    I.pf[0] = (float)I.eos.g1;
    I.pf[1] = (float)I.eos.p1;
    I.pf[2] = (float)I.eos.gm1_1;
    I.pf[3] = (float)I.eos.gp1;
    I.pf[4] = (float)(1.0 / I.eos.gm1_1);
    I.pf[5] = (float)(1.0 / I.eos.gm1_2);
    I.pf[6] = (float)c1;
    I.pf[7] = (float)c2;
    I.pd[0] = 1.0 / I.eos.gm1_1;
    I.pd[1] = 1.0 / I.eos.gm1_2;
    I.pd[2] = c1;
    I.pd[3] = c2;
    const bool stiff = I.eos.p1 != 0.0 || (c.model == CFD_MODEL_ALLAIRE && I.eos.p2 != 0.0);
    I.flags = (c.limiter & 3) | (c.wavespeed == CFD_WS_PVRS ? MF_PVRS : 0) |
              (I.godunov ? MF_GODUNOV : 0) | (stiff ? MF_STIFF : 0);
    for (int k = 0; k < 4; ++k)
        if (c.bc[k] == CFD_BC_REFLECTIVE) I.flags |= MF_BC << k;
    I.max_steps = max_steps;
    I.active = 1;
    I.fp64 = c.precision == CFD_PREC_FP64_FAST;
    // upload: the ghosted FP64 grid (or the device-built SoA state) goes
    // through a temporary staging buffer, followed by the FP64 SoA copy the
    // initial wave-speed reduction reads
    int g = c.flux_solver == CFD_FLUX_GODUNOV ? 1 : 2;
    size_t ghosted = host_ic ? (size_t)nv * (c.nx + 2 * g) * (size_t)(c.ny + 2 * g) : 0;
    size_t soa = rs ? 0 : (size_t)nv * plane;
    double* staging = nullptr;
    cudaError_t e = rs ? cudaSuccess
                       : pool_alloc(reinterpret_cast<void**>(&staging),
                                    sizeof(double) * (ghosted + soa), b->copy);
    if (e != cudaSuccess) {
        pool_free(m.mem, b->copy);
        return cfd_fail(CFD_ERR_NOMEM, "staging: %s", cudaGetErrorString(e));
    }
    DevState init;
    memset(&init, 0, sizeof init);
    init.T = c.T;
    init.cfl = c.cfl;
    init.dx = c.dx;
    init.dy = c.dy;
    if (rs) {  // the saved time state, current state in buffer 0
        init.t = rs->h->t;
        init.dt = rs->h->dt;
        init.maxu = rs->h->maxu;
        init.maxv = rs->h->maxv;
        init.mass1 = rs->h->mass1;
        init.mass2 = rs->h->mass2;
        init.n = rs->h->n;
        init.done = rs->h->t >= c.T;
    }
    int r = CFD_OK;
    do {
        if (rs) {
            for (int w = 0; w < 2 && !e; ++w) {
                e = cudaMemcpy2DAsync(I.q4[0][w], pitch * sizeof(float4), rs->q4[w],
                                      c.nx * sizeof(float4), c.nx * sizeof(float4), c.ny,
                                      cudaMemcpyHostToDevice, b->copy);
                if (!e && nv == 6)
                    e = cudaMemcpy2DAsync(I.q2[0][w], pitch * sizeof(float2), rs->q2[w],
                                          c.nx * sizeof(float2), c.nx * sizeof(float2), c.ny,
                                          cudaMemcpyHostToDevice, b->copy);
            }
            if (!e) e = cudaMemcpyAsync(I.st, &init, sizeof init, cudaMemcpyHostToDevice, b->copy);
            if (!e) e = cudaStreamSynchronize(b->copy);
            if (e) r = cfd_fail(CFD_ERR_CUDA, "restore: %s", cudaGetErrorString(e));
            break;
        }
        if ((e = cudaMemcpyAsync(I.st, &init, sizeof init, cudaMemcpyHostToDevice, b->copy))) {
            r = cfd_fail(CFD_ERR_CUDA, "upload: %s", cudaGetErrorString(e));
            break;
        }
        if (host_ic) {
            if ((e = cudaMemcpyAsync(staging, host_ic, sizeof(double) * ghosted,
                                     cudaMemcpyHostToDevice, b->copy))) {
                r = cfd_fail(CFD_ERR_CUDA, "upload: %s", cudaGetErrorString(e));
                break;
            }
            ghosted_to_mixed<<<148 * 4, 256, 0, b->copy>>>(staging, I, staging + ghosted, g);
        } else {
            cfdic::Geom geo{c.x0, c.y0, c.dx, c.dy};
            if ((e = cfdic::build_device(*prog, *prog_eos, geo, c.nx, c.ny, staging,
                                         (long long)plane, pitch, b->copy))) {
                r = cfd_fail(CFD_ERR_CUDA, "initial condition: %s", cudaGetErrorString(e));
                break;
            }
            soa_to_mixed<<<148 * 4, 256, 0, b->copy>>>(staging, I);
        }
        if (c.model == CFD_MODEL_EULER)
            init_reduce<MODEL_EULER><<<kInitBlocks, 256, 0, b->copy>>>(
                staging + ghosted, (long long)plane, pitch, c.nx, c.ny, I.eos, I.st, I.partials);
        else
            init_reduce<MODEL_ALLAIRE><<<kInitBlocks, 256, 0, b->copy>>>(
                staging + ghosted, (long long)plane, pitch, c.nx, c.ny, I.eos, I.st, I.partials);
        // no synchronisation: the pageable source has been read when the copy
        // call returns, and everything else is ordered on the batch stream
        if ((e = cudaGetLastError())) {
            r = cfd_fail(CFD_ERR_CUDA, "upload kernels: %s", cudaGetErrorString(e));
            break;
        }
    } while (0);
    pool_free(staging, b->copy);
    if (r) {
        pool_free(m.mem, b->copy);
        return r;
    }
    cudaEvent_t done_ev;
    if (cudaEventCreateWithFlags(&done_ev, cudaEventDisableTiming) != cudaSuccess ||
        cudaEventRecord(done_ev, b->copy) != cudaSuccess) {
        cudaStreamSynchronize(b->copy);  // fall back to waiting here
    } else {
        b->pending.push_back(done_ev);
    }
    b->used += bytes;
    b->members.push_back(m);
    b->dirty = true;
    *id_out = m.id;
    return CFD_OK;
}

int cfd_batch_add(cfd_batch* b, const cfd_config* cfg, const double* host_ic, int max_steps,
                  int* id_out) {
    if (!b || !cfg || !host_ic || !id_out) return cfd_fail(CFD_ERR_INVALID, "null argument");
    return add_member(b, cfg, host_ic, nullptr, nullptr, max_steps, id_out);
}

int cfd_batch_add_recipe(cfd_batch* b, const cfd_config* cfg, int recipe, uint64_t seed,
                         int nbubbles, int max_steps, int* id_out) {
    if (!b || !cfg || !id_out) return cfd_fail(CFD_ERR_INVALID, "null argument");
    std::vector<cfdic::Op> ops;
    cfdic::Eos q;
    int r = cfdic::recipe_program(cfg, recipe, seed, nbubbles, ops, q);
    if (r) return cfd_fail(r, "recipe %d does not apply to this configuration", recipe);
    return add_member(b, cfg, nullptr, &ops, &q, max_steps, id_out);
}

static Member* find(cfd_batch* b, int id) {
    for (auto& m : b->members)
        if (m.id == id) return &m;
    return nullptr;
}

int cfd_batch_remove(cfd_batch* b, int id) {
    if (!b) return cfd_fail(CFD_ERR_INVALID, "null batch");
    if (int r = wait_uploads(b)) return r;
    for (size_t i = 0; i < b->members.size(); ++i)
        if (b->members[i].id == id) {
            pool_free(b->members[i].mem, b->stream);  // after the work queued so far
            b->used -= b->members[i].bytes;
            b->members.erase(b->members.begin() + i);
            b->dirty = true;
            return CFD_OK;
        }
    return cfd_fail(CFD_ERR_INVALID, "no instance %d", id);
}

int cfd_batch_size(cfd_batch* b, int* count, size_t* used, size_t* budget) {
    if (!b) return cfd_fail(CFD_ERR_INVALID, "null batch");
    if (count) *count = (int)b->members.size();
    if (used) *used = b->used;
    if (budget) *budget = b->budget;
    return CFD_OK;
}

int cfd_batch_set_shapes(cfd_batch* b, int model, int shape_x, int shape_y) {
    if (!b || model < 0 || model > 1 || shape_x < 0 || shape_x >= kNumShapesX || shape_y < 0 ||
        shape_y >= kNumShapesY)
        return cfd_fail(CFD_ERR_INVALID, "bad shape selection");
    b->shape[model][DIR_X] = shape_x;
    b->shape[model][DIR_Y] = shape_y;
    b->dirty = true;
    b->tuned = true;
    return CFD_OK;
}

int cfd_batch_get_shapes(cfd_batch* b, int model, int* shape_x, int* shape_y) {
    if (!b || model < 0 || model > 1) return cfd_fail(CFD_ERR_INVALID, "bad arguments");
    if (shape_x) *shape_x = b->shape[model][DIR_X];
    if (shape_y) *shape_y = b->shape[model][DIR_Y];
    return CFD_OK;
}

int cfd_batch_set_march_rows(cfd_batch* b, int model, int rows) {
    if (!b || model < 0 || model > 1 || (rows != 0 && (rows < kMarchMinRows || rows > kMarchMaxRows)))
        return cfd_fail(CFD_ERR_INVALID, "bad strip length (0 or %d..%d)", kMarchMinRows,
                        kMarchMaxRows);
    b->march_fixed[model] = rows;
    b->dirty = true;
    return CFD_OK;
}

int cfd_batch_get_march_rows(cfd_batch* b, int model, int* rows) {
    if (!b || model < 0 || model > 1 || !rows) return cfd_fail(CFD_ERR_INVALID, "bad arguments");
    if (int r = build_tables(b)) return r;
    *rows = b->march_used[model];
    return CFD_OK;
}

int cfd_batch_get_segment_rows(cfd_batch* b, int model, int precision, int* rows) {
    if (!b || model < 0 || model > 1 || !rows ||
        (precision != CFD_PREC_MIXED && precision != CFD_PREC_FP64_FAST))
        return cfd_fail(CFD_ERR_INVALID, "bad arguments");
    if (int r = build_tables(b)) return r;
    *rows = b->seg_used[model][precision == CFD_PREC_FP64_FAST];
    return CFD_OK;
}

// Autotuner: runs `steps_per_trial` real steps with each tile shape per model
// and sweep direction, keeps the fastest per cell (CUDA events).  The results
// of the mixed sweeps do not depend on the tiling, so the trial steps are
// ordinary steps of the solves.
int cfd_batch_autotune(cfd_batch* b, int steps_per_trial, double* best_ms) {
    if (!b) return cfd_fail(CFD_ERR_INVALID, "null batch");
    if (steps_per_trial < 1) steps_per_trial = 1;
    double best_tick = 0.0;
    for (int model = 0; model < 2; ++model) {
        bool present = false;  // the mixed form's shapes: the fast FP64 form has one each
        for (auto& m : b->members) present |= m.cfg.model == model && !m.inst.fp64;
        if (!present) continue;
        for (int dir = 0; dir < 2; ++dir) {
            double best = 1e300;
            int best_s = b->shape[model][dir];
            const int nshapes = dir == DIR_X ? kNumShapesX : kNumShapesY;
            for (int s = 0; s < nshapes; ++s) {
                b->shape[model][dir] = s;
                b->dirty = true;
                int r = build_tables(b);
                if (r) return r;
                std::vector<Timed> ev;
                for (int k = 0; k < steps_per_trial; ++k)
                    if ((r = enqueue_tick(b, &ev))) return r;
                BTRY(cudaStreamSynchronize(b->stream));
                double ms = 0.0;
                for (auto& t : ev) {
                    const auto& g = b->groups[t.group];
                    if (g.model == model && !g.fp64 && g.dir == dir) {
                        float m = 0.f;
                        cudaEventElapsedTime(&m, t.e0, t.e1);
                        ms += m;
                    }
                    cudaEventDestroy(t.e0);
                    cudaEventDestroy(t.e1);
                }
                ms /= steps_per_trial;
                if (ms < best) {
                    best = ms;
                    best_s = s;
                }
            }
            b->shape[model][dir] = best_s;
            b->dirty = true;
            best_tick += best;
        }
    }
    b->tuned = true;
    if (best_ms) *best_ms = best_tick;
    return build_tables(b);
}

// Marks members a gather found done as finished: they leave the tile lists.
static void mark_final(cfd_batch* b, const Gather& g) {
    for (size_t i = 0; i < g.ids.size(); ++i) {
        if (!g.h[i].done) continue;
        Member* m = find(b, g.ids[i]);
        if (m && !m->final) {
            m->final = true;
            b->dirty = true;
        }
    }
}

// Reads the asynchronous status gathers of cfd_batch_step and takes the
// members they found done out of the tile lists: the one whose slot the
// next chunk reuses is waited for (it follows the chunk before last, so the
// last chunk keeps the GPU busy meanwhile and the host never runs more than
// two chunks ahead); the other only if it has completed.
static int take_async_status(cfd_batch* b) {
    Gather& old = b->async[b->async_next];
    if (old.pending) {
        BTRY(cudaEventSynchronize(old.ev));
        old.pending = false;
        mark_final(b, old);
    }
    Gather& last = b->async[b->async_next ^ 1];
    if (last.pending && cudaEventQuery(last.ev) == cudaSuccess) {
        last.pending = false;
        mark_final(b, last);
    }
    return CFD_OK;
}

// Queues a status gather of every member and its copy to pinned memory.
static int issue_gather(cfd_batch* b, Gather& g) {
    const int n = (int)b->members.size();
    if (g.pending || n == 0) return CFD_OK;
    if (int r = build_tables(b)) return r;  // the device descriptors follow the membership
    if (!g.ev) BTRY(cudaEventCreateWithFlags(&g.ev, cudaEventDisableTiming));
    if (n > g.cap) {
        pool_free(g.d, b->stream);
        g.d = nullptr;
        if (g.h) {
            BTRY(cudaStreamSynchronize(b->stream));
            cudaFreeHost(g.h);
            g.h = nullptr;
        }
        int c = std::max(64, 2 * n);
        BTRY(pool_alloc(reinterpret_cast<void**>(&g.d), sizeof(PollRec) * c, b->stream));
        BTRY(cudaHostAlloc(reinterpret_cast<void**>(&g.h), sizeof(PollRec) * c,
                           cudaHostAllocDefault));
        g.cap = c;
    }
    gather_status<<<(n + 127) / 128, 128, 0, b->stream>>>(b->d_insts, n, g.d);
    BTRY(cudaGetLastError());
    BTRY(cudaMemcpyAsync(g.h, g.d, sizeof(PollRec) * n, cudaMemcpyDeviceToHost, b->stream));
    BTRY(cudaEventRecord(g.ev, b->stream));
    g.ids.resize(n);
    for (int i = 0; i < n; ++i) g.ids[i] = b->members[i].id;
    g.pending = true;
    return CFD_OK;
}

static int issue_async_status(cfd_batch* b) {
    int r = issue_gather(b, b->async[b->async_next]);
    b->async_next ^= 1;
    return r;
}

int cfd_batch_step(cfd_batch* b, int ticks) {
    if (!b) return cfd_fail(CFD_ERR_INVALID, "null batch");
    if (ticks <= 0 || b->members.empty()) return CFD_OK;
    const int K = 8;            // ticks per captured graph
    const int kCheck = 64;      // ticks between status gathers
    int r;
    for (int done_ticks = 0; done_ticks < ticks;) {
        if ((r = take_async_status(b))) return r;
        if ((r = build_tables(b))) return r;
        if (b->groups.empty()) break;  // every member has finished
        const int chunk = std::min(kCheck, ticks - done_ticks);
        if (chunk >= K) {
            if (!b->graph) {
                BTRY(cudaStreamBeginCapture(b->stream, cudaStreamCaptureModeThreadLocal));
                int rr = CFD_OK;
                for (int i = 0; i < K && rr == CFD_OK; ++i) rr = enqueue_tick(b, nullptr);
                cudaGraph_t gph;
                cudaError_t e = cudaStreamEndCapture(b->stream, &gph);
                if (rr) return rr;
                if (e != cudaSuccess) return cfd_fail(CFD_ERR_CUDA, "capture: %s", cudaGetErrorString(e));
                e = cudaGraphInstantiate(&b->graph, gph, 0);
                cudaGraphDestroy(gph);
                if (e != cudaSuccess)
                    return cfd_fail(CFD_ERR_CUDA, "instantiate: %s", cudaGetErrorString(e));
                b->graph_steps = K;
            }
            for (int i = 0; i + K <= chunk; i += K) BTRY(cudaGraphLaunch(b->graph, b->stream));
        }
        for (int i = 0; i < chunk % K; ++i)
            if ((r = enqueue_tick(b, nullptr))) return r;
        done_ticks += chunk;
        if (done_ticks < ticks && (r = issue_async_status(b))) return r;
    }
    return CFD_OK;
}

int cfd_batch_step_timed(cfd_batch* b, int ticks, double* ms_x, double* ms_y, int* launches) {
    if (!b) return cfd_fail(CFD_ERR_INVALID, "null batch");
    int r = build_tables(b);
    if (r) return r;
    std::vector<Timed> ev;
    for (int i = 0; i < ticks; ++i)
        if ((r = enqueue_tick(b, &ev))) return r;
    BTRY(cudaStreamSynchronize(b->stream));
    double sx = 0, sy = 0;
    for (auto& t : ev) {
        float m = 0.f;
        cudaEventElapsedTime(&m, t.e0, t.e1);
        if (b->groups[t.group].dir == DIR_X) sx += m;
        else sy += m;
        cudaEventDestroy(t.e0);
        cudaEventDestroy(t.e1);
    }
    if (ms_x) *ms_x = sx;
    if (ms_y) *ms_y = sy;
    if (launches) *launches = (int)ev.size();
    return CFD_OK;
}

int cfd_batch_status(cfd_batch* b, int id, cfd_status* out) {
    if (!b || !out) return cfd_fail(CFD_ERR_INVALID, "null argument");
    Member* m = find(b, id);
    if (!m) return cfd_fail(CFD_ERR_INVALID, "no instance %d", id);
    if (int r = wait_uploads(b)) return r;
    DevState d;
    BTRY(cudaMemcpyAsync(&d, m->inst.st, sizeof d, cudaMemcpyDeviceToHost, b->stream));
    BTRY(cudaStreamSynchronize(b->stream));
    memset(out, 0, sizeof *out);
    out->n = d.n;
    out->done = d.done || d.n >= m->max_steps;
    if (out->done) m->final = true;
    out->t = d.t;
    out->dt_next = d.dt;
    out->maxu = d.maxu;
    out->maxv = d.maxv;
    out->mass1 = d.mass1;
    out->mass2 = d.mass2;
    return CFD_OK;
}

// Status of every member in one device-to-host copy: ids, steps taken and a
// done flag per member (arrays of `cap` entries); returns the count.
int cfd_batch_poll(cfd_batch* b, int cap, int* ids, int* steps, int* done, double* t, int* count) {
    if (!b || !count) return cfd_fail(CFD_ERR_INVALID, "null argument");
    int n = (int)b->members.size();
    *count = n;
    if (n == 0) return CFD_OK;
    int r = build_tables(b);  // the device descriptor array follows the membership
    if (r) return r;
    if (n > b->poll_cap) {
        pool_free(b->d_poll, b->stream);
        b->d_poll = nullptr;
        if (b->h_poll) {
            BTRY(cudaStreamSynchronize(b->stream));
            cudaFreeHost(b->h_poll);
            b->h_poll = nullptr;
        }
        int c = std::max(64, 2 * n);
        BTRY(pool_alloc(reinterpret_cast<void**>(&b->d_poll), sizeof(PollRec) * c, b->stream));
        BTRY(cudaHostAlloc(reinterpret_cast<void**>(&b->h_poll), sizeof(PollRec) * c,
                           cudaHostAllocDefault));
        b->poll_cap = c;
    }
    gather_status<<<(n + 127) / 128, 128, 0, b->stream>>>(b->d_insts, n, b->d_poll);
    BTRY(cudaGetLastError());
    BTRY(cudaMemcpyAsync(b->h_poll, b->d_poll, sizeof(PollRec) * n, cudaMemcpyDeviceToHost,
                         b->stream));
    BTRY(cudaStreamSynchronize(b->stream));
    for (int i = 0; i < n && i < cap; ++i) {
        if (ids) ids[i] = b->members[i].id;
        if (steps) steps[i] = b->h_poll[i].n;
        if (done) done[i] = b->h_poll[i].done;
        if (b->h_poll[i].done) b->members[i].final = true;
        if (t) t[i] = b->h_poll[i].t;
    }
    return CFD_OK;
}

int cfd_batch_poll_issue(cfd_batch* b) {
    if (!b) return cfd_fail(CFD_ERR_INVALID, "null batch");
    if (b->issued.pending) return cfd_fail(CFD_ERR_INVALID, "a status read is already issued");
    return issue_gather(b, b->issued);
}

int cfd_batch_poll_collect(cfd_batch* b, int cap, int* ids, int* steps, int* done, double* t,
                           int* count) {
    if (!b || !count) return cfd_fail(CFD_ERR_INVALID, "null argument");
    *count = 0;
    Gather& g = b->issued;
    if (!g.pending) return CFD_OK;
    BTRY(cudaEventSynchronize(g.ev));
    g.pending = false;
    const int n = (int)g.ids.size();
    *count = n;
    for (int i = 0; i < n && i < cap; ++i) {
        if (ids) ids[i] = g.ids[i];
        if (steps) steps[i] = g.h[i].n;
        if (done) done[i] = g.h[i].done;
        if (t) t[i] = g.h[i].t;
    }
    mark_final(b, g);
    return CFD_OK;
}

int cfd_batch_save(cfd_batch* b, int id, const char* path) {
    if (!b || !path) return cfd_fail(CFD_ERR_INVALID, "null argument");
    Member* m = find(b, id);
    if (!m) return cfd_fail(CFD_ERR_INVALID, "no instance %d", id);
    if (int r = wait_uploads(b)) return r;
    const cfd_config& c = m->cfg;
    const Inst& I = m->inst;
    DevState d;
    BTRY(cudaMemcpyAsync(&d, I.st, sizeof d, cudaMemcpyDeviceToHost, b->stream));
    BTRY(cudaStreamSynchronize(b->stream));
    const int cur = d.cur & 1, nv = I.nv;
    const size_t cells = (size_t)c.nx * c.ny;
    std::vector<float4> q4[2];
    std::vector<float2> q2[2];
    for (int w = 0; w < 2; ++w) {
        q4[w].resize(cells);
        BTRY(cudaMemcpy2DAsync(q4[w].data(), c.nx * sizeof(float4), I.q4[cur][w],
                               I.pitch * sizeof(float4), c.nx * sizeof(float4), c.ny,
                               cudaMemcpyDeviceToHost, b->stream));
        if (nv == 6) {
            q2[w].resize(cells);
            BTRY(cudaMemcpy2DAsync(q2[w].data(), c.nx * sizeof(float2), I.q2[cur][w],
                                   I.pitch * sizeof(float2), c.nx * sizeof(float2), c.ny,
                                   cudaMemcpyDeviceToHost, b->stream));
        }
    }
    BTRY(cudaStreamSynchronize(b->stream));
    // packed cells -> planes: FP64 members nv planes of doubles; mixed
    // members the values of components 0..nv-1, then their compensations
    std::vector<double> planes64(I.fp64 ? nv * cells : 0);
    for (size_t q = 0; I.fp64 && q < cells; ++q) {
        double v[6];
        memcpy(v, &q4[0][q], 16);
        memcpy(v + 2, &q4[1][q], 16);
        if (nv == 6) {
            memcpy(v + 4, &q2[0][q], 8);
            memcpy(v + 5, &q2[1][q], 8);
        }
        for (int k = 0; k < nv; ++k) planes64[k * cells + q] = v[k];
    }
    std::vector<float> planes(I.fp64 ? 0 : 2 * nv * cells);
    for (int w = 0; w < 2 && !I.fp64; ++w)
        for (size_t q = 0; q < cells; ++q) {
            float* p = planes.data() + (size_t)w * nv * cells + q;
            p[0] = q4[w][q].x;
            p[cells] = q4[w][q].y;
            p[2 * cells] = q4[w][q].z;
            p[3 * cells] = q4[w][q].w;
            if (nv == 6) {
                p[4 * cells] = q2[w][q].x;
                p[5 * cells] = q2[w][q].y;
            }
        }
    CkptHeader h;
    ckpt_init(h);
    h.cfg = c;
    h.cfg.stream = nullptr;
    h.cfg.precision = I.fp64 ? CFD_PREC_FP64_FAST : CFD_PREC_MIXED;
    h.nv = nv;
    h.g = c.flux_solver == CFD_FLUX_GODUNOV ? 1 : 2;
    h.n = d.n;
    h.done = d.done;
    h.t = d.t;
    h.dt = d.dt;
    h.maxu = d.maxu;
    h.maxv = d.maxv;
    h.mass1 = d.mass1;
    h.mass2 = d.mass2;
    h.max_steps = m->max_steps;
    h.state_bytes = sizeof(float) * planes.size() + sizeof(double) * planes64.size();
    FILE* f = fopen(path, "wb");
    if (!f) return cfd_fail(CFD_ERR_INVALID, "cannot write %s", path);
    bool ok = fwrite(&h, sizeof h, 1, f) == 1 &&
              fwrite(planes.data(), sizeof(float), planes.size(), f) == planes.size() &&
              fwrite(planes64.data(), sizeof(double), planes64.size(), f) == planes64.size();
    ok = (fclose(f) == 0) && ok;
    return ok ? CFD_OK : cfd_fail(CFD_ERR_INVALID, "short write to %s", path);
}

int cfd_batch_restore(cfd_batch* b, const char* path, int max_steps, int* id_out) {
    if (!b || !path || !id_out) return cfd_fail(CFD_ERR_INVALID, "null argument");
    FILE* f = fopen(path, "rb");
    if (!f) return cfd_fail(CFD_ERR_INVALID, "cannot open %s", path);
    CkptHeader h;
    int r = ckpt_read_header(f, h);
    const int nv = h.nv;
    const size_t cells = r ? 0 : (size_t)h.cfg.nx * h.cfg.ny;
    const bool f64 = h.cfg.precision == CFD_PREC_FP64_FAST;
    if (!r && ((h.cfg.precision != CFD_PREC_MIXED && !f64) || h.cfg.model != (nv == 4 ? 0 : 1) ||
               h.state_bytes != (f64 ? sizeof(double) * nv * cells : sizeof(float) * 2 * nv * cells)))
        r = CFD_ERR_INVALID;
    std::vector<float> planes;
    std::vector<double> planes64;
    if (!r) {
        if (f64) {
            planes64.resize(nv * cells);
            if (fread(planes64.data(), sizeof(double), planes64.size(), f) != planes64.size())
                r = CFD_ERR_INVALID;
        } else {
            planes.resize(2 * nv * cells);
            if (fread(planes.data(), sizeof(float), planes.size(), f) != planes.size())
                r = CFD_ERR_INVALID;
        }
    }
    fclose(f);
    if (r) return cfd_fail(r, "%s is not a batch member checkpoint", path);
    // planes -> packed cells (the FP64 form's doubles in the same bytes)
    std::vector<float4> q4[2];
    std::vector<float2> q2[2];
    for (int w = 0; w < 2; ++w) {
        q4[w].resize(cells);
        if (nv == 6) q2[w].resize(cells);
        for (size_t q = 0; q < cells; ++q) {
            if (f64) {
                const double v[2] = {planes64[(2 * w) * cells + q], planes64[(2 * w + 1) * cells + q]};
                memcpy(&q4[w][q], v, 16);
                if (nv == 6) memcpy(&q2[w][q], &planes64[(4 + w) * cells + q], 8);
                continue;
            }
            const float* p = planes.data() + (size_t)w * nv * cells + q;
            q4[w][q] = make_float4(p[0], p[cells], p[2 * cells], p[3 * cells]);
            if (nv == 6) q2[w][q] = make_float2(p[4 * cells], p[5 * cells]);
        }
    }
    Restore rs;
    rs.h = &h;
    for (int w = 0; w < 2; ++w) {
        rs.q4[w] = q4[w].data();
        rs.q2[w] = nv == 6 ? q2[w].data() : nullptr;
    }
    cfd_config c = h.cfg;
    c.stream = nullptr;
    return add_member(b, &c, nullptr, nullptr, nullptr, max_steps < 0 ? h.max_steps : max_steps,
                      id_out, &rs);
}

int cfd_batch_download(cfd_batch* b, int id, double* host, int layout) {
    if (!b || !host) return cfd_fail(CFD_ERR_INVALID, "null argument");
    Member* m = find(b, id);
    if (!m) return cfd_fail(CFD_ERR_INVALID, "no instance %d", id);
    const cfd_config& c = m->cfg;
    // On the copy stream: a member seen done is no longer written by the
    // sweeps, so its copy overlaps them; otherwise it waits for the work
    // queued on the batch stream so far.
    if (int r = wait_uploads(b)) return r;
    if (!m->final) {
        cudaEvent_t ev;
        BTRY(cudaEventCreateWithFlags(&ev, cudaEventDisableTiming));
        cudaError_t e = cudaEventRecord(ev, b->stream);
        if (e == cudaSuccess) e = cudaStreamWaitEvent(b->copy, ev, 0);
        cudaEventDestroy(ev);
        if (e != cudaSuccess) return cfd_fail(CFD_ERR_CUDA, "download: %s", cudaGetErrorString(e));
    }
    const int cur = -1;  // read on the device
    int nv = cfd_nvar(c.model), g = c.flux_solver == CFD_FLUX_GODUNOV ? 1 : 2;
    size_t elems = layout == CFD_LAYOUT_GHOSTED_AOS
                       ? (size_t)nv * (c.nx + 2 * g) * (size_t)(c.ny + 2 * g)
                       : (size_t)nv * c.nx * c.ny;
    double* tmp = nullptr;
    BTRY(pool_alloc(reinterpret_cast<void**>(&tmp), sizeof(double) * elems, b->copy));
    int im = c.model == CFD_MODEL_EULER ? 1 : 2;
    if (layout == CFD_LAYOUT_GHOSTED_AOS)
        mixed_to_ghosted<<<148 * 4, 256, 0, b->copy>>>(m->inst, cur, tmp, g, im, im + 1, 1);
    else  // interior only, AoS; reordered to SoA planes below
        mixed_to_ghosted<<<148 * 4, 256, 0, b->copy>>>(m->inst, cur, tmp, 0, -1, -1, 0);
    cudaError_t e = cudaGetLastError();
    if (e == cudaSuccess)
        e = cudaMemcpyAsync(host, tmp, sizeof(double) * elems, cudaMemcpyDeviceToHost, b->copy);
    if (e == cudaSuccess) e = cudaStreamSynchronize(b->copy);
    pool_free(tmp, b->copy);
    if (e != cudaSuccess) return cfd_fail(CFD_ERR_CUDA, "download: %s", cudaGetErrorString(e));
    if (layout == CFD_LAYOUT_SOA) {
        // the kernel wrote AoS interior; reorder to SoA planes on the host
        std::vector<double> aos(host, host + elems);
        size_t cells = (size_t)c.nx * c.ny;
        for (size_t q = 0; q < cells; ++q)
            for (int k = 0; k < nv; ++k) host[k * cells + q] = aos[q * nv + k];
    }
    return CFD_OK;
}

}  // extern "C"
