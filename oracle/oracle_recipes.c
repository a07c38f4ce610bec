/* Seeded workload recipes (four-quadrant Riemann problem, shock + bubbles,
 * water shock on an air bubble) restated for the CPU side.  TEST
 * INFRASTRUCTURE ONLY: bench.py's reference arm and CPU baseline build their
 * initial grids here, so that the reference's timed loop (oracle/_ref) runs
 * without the shipped library loaded, and the tests check that these grids
 * equal the library's host builder (cfd_recipe_ic) bit for bit.
 *
 * The reference has no seeded recipes; the shapes are its set_ICs helpers:
 * sub-sampled circles (E/sourcecode/euler_io.cpp:392-433,
 * A/sourcecode/allaire_diffuse_io.cpp:358-399) and half spaces
 * (A/sourcecode/allaire_diffuse_io.cpp:312-355), the state conversions of
 * E/headers/misc_euler.hpp:63-97 and A/headers/misc.hpp:130-163, cell centres
 * of E/headers/sim_info.hpp:40-46.  Random numbers: the 64-bit Mersenne
 * twister MT19937-64 (Matsumoto and Nishimura, 2000; the C++ library's
 * std::mt19937_64), top 53 bits scaled to [0, 1).
 */
#include <math.h>
#include <stdint.h>
#include <string.h>

#include "cfd_oracle.h"

enum { RECIPE_FOUR_QUADRANT = 0, RECIPE_SHOCK_BUBBLES = 1, RECIPE_WATER_SHOCK_AIR_BUBBLE = 2 };

/* ------------------------------------------------------- MT19937-64 --- */
#define MT_N 312
#define MT_M 156
typedef struct {
    uint64_t s[MT_N];
    int i;
} mt64;

static void mt_seed(mt64* m, uint64_t seed) {
    m->s[0] = seed;
    for (int k = 1; k < MT_N; ++k)
        m->s[k] = 6364136223846793005ULL * (m->s[k - 1] ^ (m->s[k - 1] >> 62)) + (uint64_t)k;
    m->i = MT_N;
}

static uint64_t mt_next(mt64* m) {
    const uint64_t upper = 0xFFFFFFFF80000000ULL, lower = 0x7FFFFFFFULL;
    const uint64_t a = 0xB5026F5AA96619E9ULL;
    if (m->i >= MT_N) {
        for (int k = 0; k < MT_N; ++k) {
            uint64_t x = (m->s[k] & upper) | (m->s[(k + 1) % MT_N] & lower);
            uint64_t xa = x >> 1;
            if (x & 1ULL) xa ^= a;
            m->s[k] = m->s[(k + MT_M) % MT_N] ^ xa;
        }
        m->i = 0;
    }
    uint64_t x = m->s[m->i++];
    x ^= (x >> 29) & 0x5555555555555555ULL;
    x ^= (x << 17) & 0x71D67FFFEDA60000ULL;
    x ^= (x << 37) & 0xFFF7EEE000000000ULL;
    x ^= x >> 43;
    return x;
}

static double mt_u(mt64* m) { return (double)(mt_next(m) >> 11) * (1.0 / 9007199254740992.0); }
static double mt_range(mt64* m, double a, double b) { return a + (b - a) * mt_u(m); }

/* ------------------------------------------------- state conversions --- */
typedef struct {
    int model;
    double g1, p1, g2, p2;
} reos;

static void p2c(const reos* q, const double* W, double* U) {
    if (q->model == 0) {
        double rho = W[0], u = W[1], v = W[2], p = W[3];
        double e = (p + q->g1 * q->p1) / ((q->g1 - 1.0) * rho);
        U[0] = rho;
        U[1] = rho * u;
        U[2] = rho * v;
        U[3] = rho * e + 0.5 * rho * (u * u + v * v);
    } else {
        double rho = W[0] + W[1];
        double z = W[5];
        double eps = z / (q->g1 - 1.0) + (1.0 - z) / (q->g2 - 1.0);
        double k = (z * q->g1 * q->p1 / (q->g1 - 1.0) + (1.0 - z) * q->g2 * q->p2 / (q->g2 - 1.0)) /
                   eps;
        double e = (W[4] + k) * eps / rho;
        U[0] = W[0];
        U[1] = W[1];
        U[2] = rho * W[2];
        U[3] = rho * W[3];
        U[4] = rho * e + 0.5 * rho * (W[2] * W[2] + W[3] * W[3]);
        U[5] = W[5];
    }
}

static void c2p(const reos* q, const double* U, double* W) {
    if (q->model == 0) {
        double rho = U[0];
        double u = U[1] / rho;
        double v = U[2] / rho;
        double e = U[3] / rho - 0.5 * (u * u + v * v);
        W[0] = rho;
        W[1] = u;
        W[2] = v;
        W[3] = (q->g1 - 1.0) * rho * e - q->g1 * q->p1;
    } else {
        double rho = U[0] + U[1];
        double u = U[2] / rho, v = U[3] / rho;
        double z = U[5];
        double e = U[4] / rho - 0.5 * (u * u + v * v);
        double eps = z / (q->g1 - 1.0) + (1.0 - z) / (q->g2 - 1.0);
        double k = (z * q->g1 * q->p1 / (q->g1 - 1.0) + (1.0 - z) * q->g2 * q->p2 / (q->g2 - 1.0)) /
                   eps;
        W[0] = U[0];
        W[1] = U[1];
        W[2] = u;
        W[3] = v;
        W[4] = rho * e / eps - k;
        W[5] = z;
    }
}

/* Fraction of the N x N sample points of a cell inside a circle
 * (E/sourcecode/euler_io.cpp:300-318 with the circle test of :392-433). */
static double circle_frac(double ccx, double ccy, double dx, double dy, int N, double cx,
                          double cy, double R) {
    int inside = 0;
    double delx = dx / N, dely = dy / N;
    double blx = ccx - 0.5 * dx, bly = ccy - 0.5 * dy;
    for (int p = 0; p < N; ++p)
        for (int r = 0; r < N; ++r) {
            double sx = blx + (p + 0.5) * delx - cx;
            double sy = bly + (r + 0.5) * dely - cy;
            if (sqrt(sx * sx + sy * sy) <= R) inside++;
        }
    return (double)inside / (N * N);
}

/* Parameters of a recipe (the library's cfd_recipe_config). */
static int recipe_params(int recipe, int nx, int ny, ref_params* p, reos* q) {
    memset(p, 0, sizeof *p);
    p->nx = nx;
    p->ny = ny;
    p->gamma2 = 1.4;
    p->limiter = REF_LIM_MINMOD;
    p->flux_solver = REF_FLUX_MUSCL;
    p->splitting = REF_SPLIT_NAIVE;
    p->wavespeed = REF_WS_DAVIS;
    switch (recipe) {
        case RECIPE_FOUR_QUADRANT:
            p->gamma1 = 1.4;
            p->dx = 1.0 / nx;
            p->dy = 1.0 / ny;
            p->cfl = 0.8;
            p->T = 0.3;
            p->limiter = REF_LIM_VANLEER;
            break;
        case RECIPE_SHOCK_BUBBLES:
            p->gamma1 = 1.4;
            p->dx = 1.0 / nx;
            p->dy = 1.0 / ny;
            p->cfl = 0.8;
            p->T = INFINITY;
            p->bc[2] = p->bc[3] = 1; /* reflective bottom and top */
            break;
        case RECIPE_WATER_SHOCK_AIR_BUBBLE:
            p->gamma1 = 4.4;
            p->pinf1 = 6e8;
            p->gamma2 = 1.4;
            p->pinf2 = 0.0;
            p->dx = 2.0 / nx;
            p->dy = 1.0 / ny;
            p->cfl = 0.6;
            p->T = INFINITY;
            p->wavespeed = REF_WS_PVRS;
            p->z_min = 1e-6;
            break;
        default:
            return -1;
    }
    q->model = recipe == RECIPE_WATER_SHOCK_AIR_BUBBLE ? 1 : 0;
    q->g1 = p->gamma1;
    q->p1 = p->pinf1;
    q->g2 = p->gamma2;
    q->p2 = p->pinf2;
    return 0;
}

/* Initial ghosted grid ((ny+4) x (nx+4) cells of 4 or 6 doubles, every cell
 * ghost cells included evaluated from its centre) and parameters of a recipe.
 * Returns 0, or -1 for an unknown recipe. */
int oracle_recipe_ic(int recipe, int nx, int ny, unsigned long long seed, int nbubbles,
                     double* grid, ref_params* p_out) {
    ref_params p;
    reos q;
    if (recipe_params(recipe, nx, ny, &p, &q)) return -1;
    const int g = 2, nv = q.model == 0 ? 4 : 6;
    const int rows = ny + 2 * g, cols = nx + 2 * g;
    const double dx = p.dx, dy = p.dy;
#define CELL(i, j) (grid + ((size_t)(i) * cols + (j)) * nv)
#define CCX(j) (p.x0 + (double)((j) - g) * dx + 0.5 * dx)
#define CCY(i) (p.y0 + (double)((i) - g) * dy + 0.5 * dy)
    if (recipe == RECIPE_FOUR_QUADRANT) {
        const double Wq[4][4] = {{1.5, 0.0, 0.0, 1.5},
                                 {0.5323, 1.206, 0.0, 0.3},
                                 {0.138, 1.206, 1.206, 0.029},
                                 {0.5323, 0.0, 1.206, 0.3}};
        double Uq[4][4];
        for (int k = 0; k < 4; ++k) p2c(&q, Wq[k], Uq[k]);
        for (int i = 0; i < rows; ++i)
            for (int j = 0; j < cols; ++j) {
                int right = CCX(j) > 0.5, top = CCY(i) > 0.5;
                int s = top ? (right ? 0 : 1) : (right ? 3 : 2);
                memcpy(CELL(i, j), Uq[s], sizeof(double) * 4);
            }
    } else if (recipe == RECIPE_SHOCK_BUBBLES) {
        double Wbg[4] = {1.0, 0.0, 0.0, 1.0}, Ubg[4];
        p2c(&q, Wbg, Ubg);
        for (int i = 0; i < rows; ++i)
            for (int j = 0; j < cols; ++j) memcpy(CELL(i, j), Ubg, sizeof Ubg);
        mt64 m;
        mt_seed(&m, seed);
        const double reach_pad = 2.0 * fmax(dx, dy);
        for (int b = 0; b < nbubbles; ++b) {
            double cx = mt_range(&m, 0.2, 1.0);
            double cy = mt_u(&m);
            double R = mt_range(&m, 0.02, 0.08);
            double rho = exp(mt_range(&m, log(0.1), log(10.0)));
            double Wb[4] = {rho, 0.0, 0.0, 1.0};
            /* cells farther than R + 2 max(dx, dy) hold no sample point inside */
            for (int i = 0; i < rows; ++i) {
                double ccy = CCY(i), dyc = ccy - cy;
                if (fabs(dyc) > R + reach_pad + dy) continue;
                for (int j = 0; j < cols; ++j) {
                    double ccx = CCX(j), dxc = ccx - cx;
                    if (sqrt(dxc * dxc + dyc * dyc) > R + reach_pad) continue;
                    double frac = circle_frac(ccx, ccy, dx, dy, 10, cx, cy, R);
                    if (frac == 0.0) continue;
                    double W[6];
                    c2p(&q, CELL(i, j), W);
                    for (int k = 0; k < 4; ++k) W[k] = frac * Wb[k] + (1.0 - frac) * W[k];
                    p2c(&q, W, CELL(i, j));
                }
            }
        }
        double gm = p.gamma1, M = 2.0;
        double rho2 = (gm + 1.0) * M * M / ((gm - 1.0) * M * M + 2.0);
        double p2 = 1.0 + 2.0 * gm / (gm + 1.0) * (M * M - 1.0);
        double u2 = M * sqrt(gm) * (1.0 - 1.0 / rho2);
        double Wp[4] = {rho2, u2, 0.0, p2}, Up[4];
        p2c(&q, Wp, Up);
        for (int i = 0; i < rows; ++i)
            for (int j = 0; j < cols; ++j)
                if (CCX(j) * 1.0 + CCY(i) * 0.0 <= 0.1) memcpy(CELL(i, j), Up, sizeof Up);
    } else {
        double zm = p.z_min > 0.0 ? p.z_min : 1e-6;
        double rho_w = 1000.0, rho_a = 1.0, p0 = 1e5, p1 = 1e9;
        mt64 m;
        mt_seed(&m, seed);
        double cx = mt_range(&m, 0.6, 1.4);
        double cy = mt_range(&m, 0.3, 0.7);
        double R = mt_range(&m, 0.1, 0.2);
        double zw = 1.0 - zm, za = zm;
        double Ww[6] = {zw * rho_w, (1.0 - zw) * rho_a, 0.0, 0.0, p0, zw};
        double Wa[6] = {za * rho_w, (1.0 - za) * rho_a, 0.0, 0.0, p0, za};
        for (int i = 0; i < rows; ++i)
            for (int j = 0; j < cols; ++j) {
                double frac = circle_frac(CCX(j), CCY(i), dx, dy, 10, cx, cy, R);
                double W[6];
                for (int k = 0; k < 6; ++k) W[k] = frac * Wa[k] + (1.0 - frac) * Ww[k];
                p2c(&q, W, CELL(i, j));
            }
        double gw = p.gamma1, pi = p.pinf1;
        double a1 = p0 + pi, a2 = p1 + pi;
        double ratio = ((gw + 1.0) * a2 + (gw - 1.0) * a1) / ((gw - 1.0) * a2 + (gw + 1.0) * a1);
        double rho_s = rho_w * ratio;
        double u_s = sqrt((p1 - p0) * (1.0 / rho_w - 1.0 / rho_s));
        double Ws[6] = {zw * rho_s, (1.0 - zw) * rho_a, u_s, 0.0, p1, zw}, Us[6];
        p2c(&q, Ws, Us);
        for (int i = 0; i < rows; ++i)
            for (int j = 0; j < cols; ++j)
                if (CCX(j) * 1.0 + CCY(i) * 0.0 <= 0.2) memcpy(CELL(i, j), Us, sizeof Us);
    }
#undef CELL
#undef CCX
#undef CCY
    if (p_out) *p_out = p;
    return 0;
}
