// Device builder of initial states from shape programs (ic_program.h).
#pragma once

#include <cuda_runtime.h>

#include <vector>

#include "ic_program.h"

namespace cfdic {

// Evaluates `ops` for every interior cell of an nx x ny grid into FP64 SoA
// planes (`plane` elements apart, rows `pitch` elements apart) on `stream`.
// The program is copied to stream-ordered device memory, so the host vector
// may go away when the call returns.  Returns a cudaError_t.
cudaError_t build_device(const std::vector<Op>& ops, const Eos& q, const Geom& G, int nx, int ny,
                         double* soa, long long plane, int pitch, cudaStream_t stream);

// Evaluates `ops` for every ghost cell (corners included) of the grid with
// g ghost layers, into a ghost frame (cfd_frame.h), as set_ICs fills the
// reference's ghost cells.
cudaError_t build_frame_device(const std::vector<Op>& ops, const Eos& q, const Geom& G, int nx,
                               int ny, int g, double* frame, cudaStream_t stream);

}  // namespace cfdic
