// A compute_dt entry point that allocates no device memory.
//
// Who needs it: callers that may not call cudaMalloc.  A host application or
// framework that owns every device allocation through its own pool or a
// fixed budget cannot let a library allocate behind its accounting, and a
// latency-critical loop cannot afford the device-wide synchronisation that
// cudaMalloc and cudaFree imply.  Such callers hand over the state and a
// small output buffer they already own; the reduction's per-row scratch
// lives in a fixed array compiled into this library instead.
//
// Scratch: g_noalloc_scratch, a file-scope __device__ array of
// 4 * kNoAllocMaxRows doubles (one partial per grid row: max(|u|+c),
// max(|v|+c) and the two mass sums) plus one completion counter, 256 KiB in
// all.  Every GPU that loads the library holds it until the process exits.
// Grids with more than kNoAllocMaxRows rows are rejected.
//
// Compiled with --fmad=false like the sweeps: the wave speeds and dt are
// formed exactly as the reference's compute_dt does
// (E/sourcecode/euler_timestep.cpp:7-44, A/sourcecode/allaire_diffuse_timestep.cpp:8-48).
#include <cuda_runtime.h>

#include <cstdio>
#include <cstring>
#include <mutex>

#include "../../include/cfdgpu.h"
#include "cfd_config.h"
#include "cfd_error.h"
#include "cfd_sweep.cuh"

using namespace cfd;

namespace {

constexpr int kNoAllocMaxRows = 8192;
constexpr int kScratchDoubles = 4 * kNoAllocMaxRows + 32;  // partials + counter slot

// Shared by every call on a device; keeps the last call's contents.
static __device__ __align__(256) double g_noalloc_scratch[kScratchDoubles];

struct NoAllocArgs {
    const double* state;
    long long plane;
    int pitch, nx, ny, n;
    double t, T, cfl, dx, dy;
    Eos eos;
    double* out;        // dt, maxu, maxv, mass1*dx*dy, mass2*dx*dy
    double* scratch;    // device address of g_noalloc_scratch
};

template <int MODEL>
__global__ void __launch_bounds__(256) noalloc_dt_kernel(NoAllocArgs A) {
    constexpr int NV = ModelTraits<MODEL>::NV;
    const int row = blockIdx.x;
    double mu = 0.0, mv = 0.0, m1 = 0.0, m2 = 0.0;
    for (int j = threadIdx.x; j < A.nx; j += blockDim.x) {
        double U[NV];
#pragma unroll
        for (int k = 0; k < NV; ++k) U[k] = A.state[k * A.plane + (long long)row * A.pitch + j];
        double su, sv, a, b;
        wave_speeds<MODEL>(A.eos, U, su, sv, a, b);
        mu = smax(mu, su);
        mv = smax(mv, sv);
        m1 += a;
        m2 += b;
    }
    __shared__ double red[4][8];
    __shared__ bool is_last;
    for (int o = 16; o > 0; o >>= 1) {
        mu = smax(mu, __shfl_down_sync(0xffffffffu, mu, o));
        mv = smax(mv, __shfl_down_sync(0xffffffffu, mv, o));
        m1 += __shfl_down_sync(0xffffffffu, m1, o);
        m2 += __shfl_down_sync(0xffffffffu, m2, o);
    }
    if ((threadIdx.x & 31) == 0) {
        red[0][threadIdx.x >> 5] = mu;
        red[1][threadIdx.x >> 5] = mv;
        red[2][threadIdx.x >> 5] = m1;
        red[3][threadIdx.x >> 5] = m2;
    }
    __syncthreads();
    unsigned* counter = reinterpret_cast<unsigned*>(A.scratch + 4 * kNoAllocMaxRows);
    if (threadIdx.x == 0) {
        for (int w = 1; w < 8; ++w) {
            red[0][0] = smax(red[0][0], red[0][w]);
            red[1][0] = smax(red[1][0], red[1][w]);
            red[2][0] += red[2][w];
            red[3][0] += red[3][w];
        }
        double* p = A.scratch + 4 * row;
        p[0] = red[0][0];
        p[1] = red[1][0];
        p[2] = red[2][0];
        p[3] = red[3][0];
        __threadfence();
        is_last = atomicAdd(counter, 1u) == gridDim.x - 1;
    }
    __syncthreads();
    if (!is_last || threadIdx.x != 0) return;
    __threadfence();
    // rows combined in order: reproducible mass sums
    double MU = 0.0, MV = 0.0, M1 = 0.0, M2 = 0.0;
    for (int r = 0; r < A.ny; ++r) {
        const double* p = A.scratch + 4 * r;
        MU = smax(MU, p[0]);
        MV = smax(MV, p[1]);
        M1 += p[2];
        M2 += p[3];
    }
    // E/sourcecode/euler_timestep.cpp:36-43
    double cfl = A.cfl;
    if (A.n < 5) cfl = smin(cfl, 0.2);
    double dt = cfl * smin(A.dx / MU, A.dy / MV);
    if (A.t + dt > A.T) dt = A.T - A.t;
    A.out[0] = dt;
    A.out[1] = MU;
    A.out[2] = MV;
    A.out[3] = M1 * A.dx * A.dy;
    A.out[4] = M2 * A.dx * A.dy;
    *counter = 0u;
}

std::mutex g_mu;
double* g_scratch_ptr[64] = {nullptr};

}  // namespace

extern "C" {

// See include/cfdgpu.h for the contract.
int cfd_compute_dt_noalloc(const cfd_config* cfg, const double* dev_state, int64_t plane,
                           int pitch, int n, double t, double* dev_out, void* stream) {
    if (!cfg || !dev_state || !dev_out) return cfd_fail(CFD_ERR_INVALID, "null argument");
    int r = validate_config(cfg);  // the checks cfd_create applies
    if (r) return r;
    if (pitch < cfg->nx || plane < (int64_t)pitch * cfg->ny)
        return cfd_fail(CFD_ERR_INVALID, "inconsistent grid %dx%d, pitch %d, plane %lld", cfg->nx,
                        cfg->ny, pitch, (long long)plane);
    if (cfg->ny > kNoAllocMaxRows)  // the fixed scratch holds one partial per grid row
        return cfd_fail(CFD_ERR_INVALID,
                        "cfd_compute_dt_noalloc: ny = %d exceeds the fixed scratch of %d rows; "
                        "use cfd_compute_dt on a solver instead",
                        cfg->ny, kNoAllocMaxRows);
    int dev = 0;
    cudaError_t e = cudaGetDevice(&dev);
    if (e != cudaSuccess) return cfd_fail(CFD_ERR_CUDA, "cudaGetDevice: %s", cudaGetErrorString(e));
    if (dev < 0 || dev >= 64) return cfd_fail(CFD_ERR_CUDA, "device ordinal %d out of range", dev);
    double* scratch;
    {
        // First call on a device: look up the device address of the scratch
        // array with that device current (the host-side symbol is only a
        // stand-in), and load both models' kernels, so that no later call on
        // this device loads code (which takes device memory) whichever model
        // it is for.  Make this first call before any stream capture.
        std::lock_guard<std::mutex> lk(g_mu);
        if (!g_scratch_ptr[dev]) {
            void* p = nullptr;
            cudaError_t se = cudaGetSymbolAddress(&p, g_noalloc_scratch);
            if (se != cudaSuccess || !p)
                return cfd_fail(CFD_ERR_CUDA, "cudaGetSymbolAddress(scratch): %s",
                                cudaGetErrorString(se));
            cudaFuncAttributes fa;
            se = cudaFuncGetAttributes(&fa, noalloc_dt_kernel<MODEL_EULER>);
            if (se == cudaSuccess) se = cudaFuncGetAttributes(&fa, noalloc_dt_kernel<MODEL_ALLAIRE>);
            if (se != cudaSuccess)
                return cfd_fail(CFD_ERR_CUDA, "loading the kernels: %s", cudaGetErrorString(se));
            g_scratch_ptr[dev] = static_cast<double*>(p);
        }
        scratch = g_scratch_ptr[dev];
    }
    cudaStream_t st = static_cast<cudaStream_t>(stream);
    // the completion counter must start at zero
    e = cudaMemsetAsync(scratch + 4 * kNoAllocMaxRows, 0, sizeof(unsigned), st);
    if (e != cudaSuccess) return cfd_fail(CFD_ERR_CUDA, "clearing the counter: %s", cudaGetErrorString(e));
    NoAllocArgs a;
    a.state = dev_state;
    a.plane = plane;
    a.pitch = pitch;
    a.nx = cfg->nx;
    a.ny = cfg->ny;
    a.n = n;
    a.t = t;
    a.T = cfg->T;
    a.cfl = cfg->cfl;
    a.dx = cfg->dx;
    a.dy = cfg->dy;
    a.eos = make_eos(*cfg);
    a.out = dev_out;
    a.scratch = scratch;
    if (cfg->model == CFD_MODEL_EULER)
        noalloc_dt_kernel<MODEL_EULER><<<cfg->ny, 256, 0, st>>>(a);
    else
        noalloc_dt_kernel<MODEL_ALLAIRE><<<cfg->ny, 256, 0, st>>>(a);
    e = cudaGetLastError();
    if (e != cudaSuccess) return cfd_fail(CFD_ERR_CUDA, "launch: %s", cudaGetErrorString(e));
    return CFD_OK;
}

int cfd_noalloc_max_rows(void) { return kNoAllocMaxRows; }

}  // extern "C"
