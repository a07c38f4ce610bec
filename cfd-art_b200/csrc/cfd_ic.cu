// Device builder of initial states: one thread per interior cell evaluates
// the shape program (ic_program.h) and writes the FP64 SoA state, so a
// solve's initial grid is made where it is used, with no host grid and no
// host-to-device copy of the state.  Compiled with --fmad=false like the
// host side, which makes the two bit-identical.
#include "cfd_frame.h"
#include "cfd_ic.h"

namespace cfdic {
namespace {

template <int NV>
__global__ void __launch_bounds__(256)
ic_kernel(const Op* __restrict__ ops, int nops, Eos q, Geom G, int nx, int ny,
          double* __restrict__ soa, long long plane, int pitch) {
    const long long n = (long long)nx * ny;
    for (long long idx = blockIdx.x * (long long)blockDim.x + threadIdx.x; idx < n;
         idx += (long long)gridDim.x * blockDim.x) {
        const int i = (int)(idx / nx), j = (int)(idx % nx);
        double U[6];
        eval_cell_n<NV>(ops, nops, q, G, i, j, U);
        const long long o = (long long)i * pitch + j;
#pragma unroll
        for (int k = 0; k < NV; ++k) soa[k * plane + o] = U[k];
    }
}

template <int NV>
__global__ void __launch_bounds__(256)
ic_frame_kernel(const Op* __restrict__ ops, int nops, Eos q, Geom G, int nx, int ny, int g,
                double* __restrict__ frame) {
    const long long n = cfd::frame_cells(nx, ny, g);
    for (long long f = blockIdx.x * (long long)blockDim.x + threadIdx.x; f < n;
         f += (long long)gridDim.x * blockDim.x) {
        int gi, gj;
        cfd::frame_cell(f, nx, ny, g, gi, gj);
        double U[6];
        eval_cell_n<NV>(ops, nops, q, G, gi - g, gj - g, U);
#pragma unroll
        for (int k = 0; k < NV; ++k) frame[f * NV + k] = U[k];
    }
}

// Copies the program to stream-ordered device memory.
cudaError_t stage_ops(const std::vector<Op>& ops, Op** d_ops, cudaStream_t stream) {
    size_t bytes = sizeof(Op) * (ops.empty() ? 1 : ops.size());
    cudaError_t e = cudaMallocAsync(reinterpret_cast<void**>(d_ops), bytes, stream);
    if (e) return e;
    if (!ops.empty() &&
        (e = cudaMemcpyAsync(*d_ops, ops.data(), sizeof(Op) * ops.size(), cudaMemcpyHostToDevice,
                             stream))) {
        cudaFreeAsync(*d_ops, stream);
        return e;
    }
    // pageable source: the host vector has been read when the copy call returns
    return cudaSuccess;
}

}  // namespace

cudaError_t build_frame_device(const std::vector<Op>& ops, const Eos& q, const Geom& G, int nx,
                               int ny, int g, double* frame, cudaStream_t stream) {
    Op* d_ops = nullptr;
    cudaError_t e = stage_ops(ops, &d_ops, stream);
    if (e) return e;
    if (q.model == 0)
        ic_frame_kernel<4><<<148, 256, 0, stream>>>(d_ops, (int)ops.size(), q, G, nx, ny, g, frame);
    else
        ic_frame_kernel<6><<<148, 256, 0, stream>>>(d_ops, (int)ops.size(), q, G, nx, ny, g, frame);
    e = cudaGetLastError();
    cudaError_t f = cudaFreeAsync(d_ops, stream);
    return e ? e : f;
}

cudaError_t build_device(const std::vector<Op>& ops, const Eos& q, const Geom& G, int nx, int ny,
                         double* soa, long long plane, int pitch, cudaStream_t stream) {
    Op* d_ops = nullptr;
    cudaError_t e = stage_ops(ops, &d_ops, stream);
    if (e) return e;
    long long cells = (long long)nx * ny;
    int blocks = (int)std::min<long long>((cells + 255) / 256, 148LL * 8);
    if (q.model == 0)
        ic_kernel<4><<<blocks, 256, 0, stream>>>(d_ops, (int)ops.size(), q, G, nx, ny, soa, plane,
                                                 pitch);
    else
        ic_kernel<6><<<blocks, 256, 0, stream>>>(d_ops, (int)ops.size(), q, G, nx, ny, soa, plane,
                                                 pitch);
    e = cudaGetLastError();
    cudaError_t f = cudaFreeAsync(d_ops, stream);
    return e ? e : f;
}

}  // namespace cfdic
