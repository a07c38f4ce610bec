// Binary checkpoint format of a solve (little-endian, as the host writes it):
//   CkptHeader
//   state: plain and fast FP64 solves: nv planes of nx*ny doubles
//          (row-major, no padding); mixed solves: nv planes of nx*ny floats
//          (values), then nv planes of their compensation words
//   ghost frame (has_frame): cells x nv doubles (cfd_frame.h order)
// The header keeps the solve's configuration (stream pointer cleared) and its
// device time-loop state, so a restored solve continues bit for bit as if it
// had never stopped.
#pragma once

#include <stdint.h>
#include <stdio.h>
#include <string.h>

#include "../../include/cfdgpu.h"

namespace cfd {

struct CkptHeader {
    char magic[8];          // "CFDCKPT\0"
    uint32_t version;       // 1
    uint32_t header_bytes;  // sizeof(CkptHeader)
    cfd_config cfg;         // stream = NULL
    int32_t nv, g;
    int32_t n, done;
    double t, dt, maxu, maxv, mass1, mass2;
    unsigned long long counters[8];
    int32_t has_frame;
    int32_t max_steps;      // batch members: the step limit they were added with
    uint64_t state_bytes, frame_bytes;
};

inline void ckpt_init(CkptHeader& h) {
    memset(&h, 0, sizeof h);
    memcpy(h.magic, "CFDCKPT", 8);
    h.version = 1;
    h.header_bytes = sizeof(CkptHeader);
}

// Reads and checks a header; returns CFD_OK or CFD_ERR_INVALID.
inline int ckpt_read_header(FILE* f, CkptHeader& h) {
    if (fread(&h, sizeof h, 1, f) != 1) return CFD_ERR_INVALID;
    if (memcmp(h.magic, "CFDCKPT", 8) != 0 || h.version != 1 ||
        h.header_bytes != sizeof(CkptHeader))
        return CFD_ERR_INVALID;
    if (h.cfg.nx < 2 || h.cfg.ny < 2 || (h.nv != 4 && h.nv != 6)) return CFD_ERR_INVALID;
    return CFD_OK;
}

}  // namespace cfd
