// Ghost frame: the ghost cells of a ghosted grid stored on their own (AoS,
// nv doubles per cell), for callers that need the ghost values the
// reference's grid holds between boundary fills.  Order: the g bottom rows
// and the g top rows (full width W = nx + 2g, corners included), then the
// g left and the g right columns of the ny interior rows.
#pragma once

#ifdef __CUDACC__
#define FRAME_HD __host__ __device__ __forceinline__
#else
#define FRAME_HD inline
#endif

namespace cfd {

FRAME_HD long long frame_cells(int nx, int ny, int g) {
    return 2LL * g * (nx + 2 * g) + 2LL * ny * g;
}

// Ghosted coordinates (row gi, column gj) of frame cell f.
FRAME_HD void frame_cell(long long f, int nx, int ny, int g, int& gi, int& gj) {
    const long long W = nx + 2 * g, rows = (long long)g * W, cols = (long long)ny * g;
    if (f < rows) {
        gi = (int)(f / W);
        gj = (int)(f % W);
    } else if (f < 2 * rows) {
        f -= rows;
        gi = ny + g + (int)(f / W);
        gj = (int)(f % W);
    } else if (f < 2 * rows + cols) {
        f -= 2 * rows;
        gi = g + (int)(f / g);
        gj = (int)(f % g);
    } else {
        f -= 2 * rows + cols;
        gi = g + (int)(f / g);
        gj = nx + g + (int)(f % g);
    }
}

FRAME_HD long long frame_index(int gi, int gj, int nx, int ny, int g) {
    const long long W = nx + 2 * g, rows = (long long)g * W, cols = (long long)ny * g;
    if (gi < g) return (long long)gi * W + gj;
    if (gi >= ny + g) return rows + (long long)(gi - ny - g) * W + gj;
    if (gj < g) return 2 * rows + (long long)(gi - g) * g + gj;
    return 2 * rows + cols + (long long)(gi - g) * g + (gj - nx - g);
}

}  // namespace cfd
