// Initial states as shape programs: an ordered list of operations that each
// set or modify the state of a cell from its centre and N x N sub-cell
// sample points.  The same per-cell evaluation runs on the host (over the
// ghosted grid, bit-identical to the reference's set_ICs) and on the device
// (over the interior, straight into the solver's buffers), so an initial
// state of any size is built on the GPU with no host grid and no
// host-to-device copy.  Both sides compile this header without contracted
// multiply-adds and with correctly rounded division and square root, so they
// agree bit for bit.
//
// Operations (reference file:line of the set_ICs helper each follows):
//   FILL          U = v[0]
//   ADD_CIRCLE    U += frac * v[0]; frac = 0 when the centre is farther than
//                 R + 2 dx from the circle centre (E/sourcecode/euler_io.cpp:335-389)
//   ADD_RECT      U += frac * v[0]                 (E/sourcecode/euler_io.cpp:282-330)
//   SET_CIRCULAR  W = frac v[0] + (1-frac) v[1]; U = p2c(W)
//                 (E/sourcecode/euler_io.cpp:392-433, A/sourcecode/allaire_diffuse_io.cpp:358-399)
//   SET_PLANAR    U = a x + b y <= c ? v[0] : v[1] (A/sourcecode/allaire_diffuse_io.cpp:312-355)
//   SET_HALFSPACE U = v[0] where a x + b y <= c
//   BLEND_CIRCLE  W = frac v[0] + (1-frac) c2p(U), U = p2c(W), cells with
//                 frac = 0 untouched (seeded bubble recipes)
//   QUADRANTS     U = v[k], k from (x > a[0], y > a[1]) (four-quadrant Riemann problem)
//   MIXED_CELL    Allaire: material 1 in its pre- or post-shock state by the
//                 cell centre's x, material 2 where N x N sub-samples fall in
//                 a rectangle or left of the sine interface
//                 x = 2.9 - 0.2 sin(2 pi (y + 1/4)) (shocked_SF6, TSTM, RMI_SF6:
//                 A/sourcecode/allaire_diffuse_io.cpp:659-870)
//   RING_CELL     Allaire: material 1 blended between an inner and an outer
//                 state by a sampled circle, material 2 outside a perturbed
//                 ring r(theta) (tin_air_implosion: A/sourcecode/allaire_diffuse_io.cpp:872-983)
// The last two call sin / cos / atan2: the host gets the C library's values,
// the device CUDA's, which agree to an ulp or so; a cell can differ only if
// one of its sample points lies that close to the interface.
#pragma once

#include <math.h>
#include <stdint.h>

#ifdef __CUDACC__
#define IC_HD __host__ __device__ __forceinline__
#else
#define IC_HD inline
#endif

namespace cfdic {

enum OpKind {
    OP_FILL = 1,
    OP_ADD_CIRCLE = 2,
    OP_ADD_RECT = 3,
    OP_SET_CIRCULAR = 4,
    OP_SET_PLANAR = 5,
    OP_SET_HALFSPACE = 6,
    OP_BLEND_CIRCLE = 7,
    OP_QUADRANTS = 8,
    OP_MIXED_CELL = 9,
    OP_RING_CELL = 10,
};

struct Op {
    int kind;
    int n;         // sub-samples per direction
    double a[4];   // circle (cx, cy, R); rectangle (blx, bly, w, h); plane (a, b, c); split (x, y)
    double v[4][6];
};

struct Eos {
    int model;  // CFD_MODEL_EULER (0) or CFD_MODEL_ALLAIRE (1)
    double g1, p1, g2, p2;
};

struct Geom {
    double x0, y0, dx, dy;
};

// E/headers/misc_euler.hpp:82-97
IC_HD void euler_p2c(const Eos& q, const double* W, double* U) {
    double rho = W[0], u = W[1], v = W[2], p = W[3];
    double e = (p + q.g1 * q.p1) / ((q.g1 - 1.0) * rho);
    U[0] = rho;
    U[1] = rho * u;
    U[2] = rho * v;
    U[3] = rho * e + 0.5 * rho * (u * u + v * v);
}

// E/headers/misc_euler.hpp:63-79
IC_HD void euler_c2p(const Eos& q, const double* U, double* W) {
    double rho = U[0];
    double u = U[1] / rho;
    double v = U[2] / rho;
    double e = U[3] / rho - 0.5 * (u * u + v * v);
    W[0] = rho;
    W[1] = u;
    W[2] = v;
    W[3] = (q.g1 - 1.0) * rho * e - q.g1 * q.p1;
}

// A/headers/mixturemodel.hpp:26-32 and A/headers/misc.hpp:149-163
IC_HD void allaire_p2c(const Eos& q, const double* W, double* U) {
    double rho = W[0] + W[1];
    double z = W[5];
    double eps = z / (q.g1 - 1.0) + (1.0 - z) / (q.g2 - 1.0);
    double k = (z * q.g1 * q.p1 / (q.g1 - 1.0) + (1.0 - z) * q.g2 * q.p2 / (q.g2 - 1.0)) / eps;
    double e = (W[4] + k) * eps / rho;
    U[0] = W[0];
    U[1] = W[1];
    U[2] = rho * W[2];
    U[3] = rho * W[3];
    U[4] = rho * e + 0.5 * rho * (W[2] * W[2] + W[3] * W[3]);
    U[5] = W[5];
}

// A/headers/misc.hpp:130-147 with A/headers/mixturemodel.hpp:18-24
IC_HD void allaire_c2p(const Eos& q, const double* U, double* W) {
    double rho = U[0] + U[1];
    double u = U[2] / rho, v = U[3] / rho;
    double z = U[5];
    double e = U[4] / rho - 0.5 * (u * u + v * v);
    double eps = z / (q.g1 - 1.0) + (1.0 - z) / (q.g2 - 1.0);
    double k = (z * q.g1 * q.p1 / (q.g1 - 1.0) + (1.0 - z) * q.g2 * q.p2 / (q.g2 - 1.0)) / eps;
    W[0] = U[0];
    W[1] = U[1];
    W[2] = u;
    W[3] = v;
    W[4] = rho * e / eps - k;
    W[5] = z;
}

// Two-material cell of given volume fraction z of material 1 (partial
// densities, momentum, energy from each material's specific energy).
IC_HD void mixed_cell(double z, double rho1, double rho2, double u, double v, double e1, double e2,
                      double* U) {
    U[0] = z * rho1;
    U[1] = (1.0 - z) * rho2;
    U[2] = u * (z * rho1 + (1.0 - z) * rho2);
    U[3] = v * (z * rho1 + (1.0 - z) * rho2);
    U[4] = z * rho1 * e1 + (1.0 - z) * rho2 * e2 + 0.5 * (z * rho1 + (1.0 - z) * rho2) * (u * u + v * v);
    U[5] = z;
}

IC_HD int nvar(const Eos& q) { return q.model == 0 ? 4 : 6; }

IC_HD void p2c(const Eos& q, const double* W, double* U) {
    if (q.model == 0) euler_p2c(q, W, U);
    else allaire_p2c(q, W, U);
}

IC_HD void c2p(const Eos& q, const double* U, double* W) {
    if (q.model == 0) euler_c2p(q, U, W);
    else allaire_c2p(q, U, W);
}

// Fraction of the N x N sample points of the cell with lower-left corner
// (blx, bly) that lie inside the shape (E/sourcecode/euler_io.cpp:300-318).
IC_HD bool inside_circle(double sx, double sy, const double* a) {
    sx -= a[0];
    sy -= a[1];
    return sqrt(sx * sx + sy * sy) <= a[2];
}
IC_HD bool inside_rect(double sx, double sy, const double* a) {
    sx -= a[0];
    sy -= a[1];
    return (0.0 <= sx) & (sx <= a[2]) & (0.0 <= sy) & (sy <= a[3]);
}
// Material-2 regions of MIXED_CELL (a[0..3] = x0, x1, y0, y1 of a closed
// rectangle, or a[0] = pi for the sine interface) and of RING_CELL
// (a[0] = pi / 2).
IC_HD bool inside_box(double sx, double sy, const double* a) {
    return sx >= a[0] && sx <= a[1] && sy >= a[2] && sy <= a[3];
}
IC_HD bool left_of_sine(double sx, double sy, const double* a) {
    double interfacex = 2.9 - 0.2 * sin(2.0 * a[0] * (sy + 0.25));
    return interfacex > sx;
}
IC_HD bool inside_ring(double sx, double sy, const double* a) {
    double theta = atan2(sy, sx);
    theta -= a[0];
    double r = 20.0 + 0.4 * cos(22 * theta) + 0.4 * cos(17 * theta) + 0.3 * cos(29 * theta);
    return sqrt(sx * sx + sy * sy) <= r;
}
IC_HD bool inside_r24(double sx, double sy, const double*) { return sqrt(sx * sx + sy * sy) <= 24.0; }

enum { REGION_CIRCLE, REGION_RECT, REGION_BOX, REGION_SINE, REGION_RING, REGION_R24 };

IC_HD bool inside_region(int region, double sx, double sy, const double* a) {
    switch (region) {
        case REGION_CIRCLE: return inside_circle(sx, sy, a);
        case REGION_RECT: return inside_rect(sx, sy, a);
        case REGION_BOX: return inside_box(sx, sy, a);
        case REGION_SINE: return left_of_sine(sx, sy, a);
        case REGION_RING: return inside_ring(sx, sy, a);
        default: return inside_r24(sx, sy, a);
    }
}

IC_HD double sample_region(const Geom& G, double ccx, double ccy, int N, int region,
                           const double* a) {
    int numinside = 0;
    double delx = G.dx / N, dely = G.dy / N;
    double blx = ccx - 0.5 * G.dx, bly = ccy - 0.5 * G.dy;
    for (int p = 0; p < N; ++p)
        for (int r = 0; r < N; ++r) {
            double sx = blx + (p + 0.5) * delx;
            double sy = bly + (r + 0.5) * dely;
            if (inside_region(region, sx, sy, a)) numinside++;
        }
    return double(numinside) / (N * N);
}

IC_HD double sample_frac(const Geom& G, double ccx, double ccy, int N, bool circle,
                         const double* a) {
    return sample_region(G, ccx, ccy, N, circle ? REGION_CIRCLE : REGION_RECT, a);
}

// State of the cell whose centre is at column offset jj and row offset ii
// from the first interior cell (negative offsets are ghost cells): the
// reference's cell centre x0 + (j - g) dx + dx/2 (headers/sim_info.hpp:40-46).
// NV = 4 (Euler) or 6 (Allaire) components.
template <int NV>
IC_HD void eval_cell_n(const Op* ops, int nops, const Eos& q, const Geom& G, int ii, int jj,
                       double* U) {
    constexpr int nv = NV;
    const double ccx = G.x0 + double(jj) * G.dx + 0.5 * G.dx;
    const double ccy = G.y0 + double(ii) * G.dy + 0.5 * G.dy;
    double W[6] = {0.0, 0.0, 0.0, 0.0, 0.0, 0.0};
    for (int k = 0; k < nv; ++k) U[k] = 0.0;
    for (int o = 0; o < nops; ++o) {
        const Op& op = ops[o];
        switch (op.kind) {
            case OP_FILL:
                for (int k = 0; k < nv; ++k) U[k] = op.v[0][k];
                break;
            case OP_ADD_CIRCLE: {
                double dxc = ccx - op.a[0], dyc = ccy - op.a[1];
                double frac = 0.0;
                if (!(sqrt(dxc * dxc + dyc * dyc) > op.a[2] + 2.0 * G.dx))
                    frac = sample_frac(G, ccx, ccy, op.n, true, op.a);
                for (int k = 0; k < nv; ++k) U[k] += frac * op.v[0][k];
                break;
            }
            case OP_ADD_RECT: {
                double frac = sample_frac(G, ccx, ccy, op.n, false, op.a);
                for (int k = 0; k < nv; ++k) U[k] += frac * op.v[0][k];
                break;
            }
            case OP_SET_CIRCULAR: {
                double frac = sample_frac(G, ccx, ccy, op.n, true, op.a);
                for (int k = 0; k < nv; ++k) W[k] = frac * op.v[0][k] + (1.0 - frac) * op.v[1][k];
                p2c(q, W, U);
                break;
            }
            case OP_SET_PLANAR: {
                const double* s = ccx * op.a[0] + ccy * op.a[1] <= op.a[2] ? op.v[0] : op.v[1];
                for (int k = 0; k < nv; ++k) U[k] = s[k];
                break;
            }
            case OP_SET_HALFSPACE:
                if (ccx * op.a[0] + ccy * op.a[1] <= op.a[2])
                    for (int k = 0; k < nv; ++k) U[k] = op.v[0][k];
                break;
            case OP_BLEND_CIRCLE: {
                // Cells whose centre is farther than R + 2 max(dx, dy) from
                // the circle's centre have no sample point inside it.
                double dxc = ccx - op.a[0], dyc = ccy - op.a[1];
                double reach = op.a[2] + 2.0 * fmax(G.dx, G.dy);
                if (sqrt(dxc * dxc + dyc * dyc) > reach) break;
                double frac = sample_frac(G, ccx, ccy, op.n, true, op.a);
                if (frac == 0.0) break;
                c2p(q, U, W);
                for (int k = 0; k < nv; ++k) W[k] = frac * op.v[0][k] + (1.0 - frac) * W[k];
                p2c(q, W, U);
                break;
            }
            case OP_QUADRANTS: {
                bool right = ccx > op.a[0], top = ccy > op.a[1];
                int s = top ? (right ? 0 : 1) : (right ? 3 : 2);
                for (int k = 0; k < nv; ++k) U[k] = op.v[s][k];
                break;
            }
            case OP_MIXED_CELL: {
                // v[0] = pre rho1, u, e1, post rho1, u, e1; v[1] = rho2, e2,
                // x threshold, +1 (pre where x > it) or -1 (pre where x < it),
                // region (REGION_BOX or REGION_SINE)
                const double* m = op.v[0];
                bool pre = op.v[1][3] > 0.0 ? ccx > op.v[1][2] : ccx < op.v[1][2];
                double rho1 = pre ? m[0] : m[3], u = pre ? m[1] : m[4], e1 = pre ? m[2] : m[5];
                double frac = sample_region(G, ccx, ccy, op.n, (int)op.v[1][4], op.a);
                if constexpr (NV == 6)
                    mixed_cell(1.0 - frac, rho1, op.v[1][0], u, 0.0, e1, op.v[1][1], U);
                break;
            }
            case OP_RING_CELL: {
                // v[0] = inner rho1, e1, outer rho1, e1; v[1] = rho2, e2
                const double* m = op.v[0];
                double ins = sample_region(G, ccx, ccy, op.n, REGION_R24, op.a);
                double rho1 = ins * m[0] + (1.0 - ins) * m[2];
                double e1 = ins * m[1] + (1.0 - ins) * m[3];
                double frac = sample_region(G, ccx, ccy, op.n, REGION_RING, op.a);
                if constexpr (NV == 6)
                    mixed_cell(1.0 - frac, rho1, op.v[1][0], 0.0, 0.0, e1, op.v[1][1], U);
                break;
            }
            default:
                break;
        }
    }
}

IC_HD void eval_cell(const Op* ops, int nops, const Eos& q, const Geom& G, int ii, int jj,
                     double* U) {
    if (q.model == 0) eval_cell_n<4>(ops, nops, q, G, ii, jj, U);
    else eval_cell_n<6>(ops, nops, q, G, ii, jj, U);
}

}  // namespace cfdic
