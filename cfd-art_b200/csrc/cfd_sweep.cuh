// Directional sweep kernels of the split finite-volume update (plain FP64).
//
// One launch updates every interior cell along one direction:
//   x-sweep  E/sourcecode/euler_rowsweep.cpp:10-95,
//            A/sourcecode/allaire_diffuse_rowsweep.cpp:10-52
//   y-sweep  E/sourcecode/euler_colsweep.cpp:10-114,
//            A/sourcecode/allaire_diffuse_colsweep.cpp:9-73
// with the ghost-cell fill that precedes each sweep
// (E/sourcecode/euler_ppsweep.cpp:7-118) synthesised while the tile is loaded,
// and, optionally, the CFL wave-speed reduction of the new state
// (E/sourcecode/euler_timestep.cpp:7-44, A/sourcecode/allaire_diffuse_timestep.cpp:8-48)
// fused into the store, finished by the last CTA, which also advances the
// device-resident time and picks the next dt.
//
// Layout in HBM: SoA, one plane per stored component, interior cells only,
// row-major with a padded pitch.  A CTA owns a tile of TS cells along the
// sweep by NA lines across it and stages TS+4 cells per line (2-cell halo
// each side) in shared memory, x fastest, so every global access is
// coalesced in both sweep directions.  Four phases, separated by barriers:
//   P1  conserved -> primitive per staged cell
//   P2  limited slope and the four extrapolated/evolved face states per cell
//   P3  HLLC flux per face
//   P4  conservative update (+ Allaire z update / Euler fix-up), store,
//       wave-speed reduction
#pragma once

#include "cfd_physics.cuh"

namespace cfd {

enum { DIR_X = 0, DIR_Y = 1 };
enum {
    CNT_UNPHYSICAL_INPUT = 0,  // stencil state failing the reference's assert
    CNT_SLOPE_ZEROED = 1,      // "Unphysical state created by slope extrapolation"
    CNT_FIRST_ORDER = 2,       // "Unphysical state created by time evolution"
    CNT_FIXUP = 3,             // Euler post-update density/energy restore
    CNT_UNPHYSICAL_OUTPUT = 4, // Allaire assert after the z update
    CNT_N = 8
};

// Device-resident time-loop state (headers/simulation.hpp:44-61).
struct DevState {
    double t;      // simulated time of the current state
    double dt;     // dt chosen for the next step from the current state
    double T;      // end time
    double cfl;
    double maxu, maxv;    // max(|u|+c), max(|v|+c) over the current state
    double mass1, mass2;  // sum of density (Allaire: partial densities)
    double dx, dy;
    int n;         // steps taken
    int done;      // t >= T: further steps are no-ops
    unsigned ticket;  // last-CTA-done counter of the reduction
    int cur;       // which of the two state buffers holds the current state
};

struct SweepArgs {
    double* bufs[2];  // the two state buffers; input = bufs[cur ^ in_sel]
    int in_sel;
    int flip_cur;     // the finishing CTA flips DevState::cur (Strang: odd sweep count)
    long long plane;  // elements between component planes
    int pitch;        // elements between rows
    int nx, ny;
    Eos eos;
    int bc_lo, bc_hi;  // reflective walls at the low/high end along the sweep
    int limiter, wavespeed, godunov;
    double z_min;
    double h_flux;    // spacing handed to the flux solver (dx; dx or dy in y)
    double h_upd;     // spacing of the conservative update
    double dt_host;   // dt when use_host_dt
    double dt_scale;  // 1 or 0.5 (Strang half steps)
    int use_host_dt;
    int reduce;       // fuse the wave-speed reduction and the time advance
    int advance_time; // the reduction closes a step: t += dt, n++
    DevState* st;
    double* partials;  // 4 per CTA
    unsigned long long* counters;
};

__device__ __forceinline__ void block_count(unsigned long long* ctr, int idx, bool flag) {
    unsigned m = __ballot_sync(0xffffffffu, flag);
    if ((threadIdx.x & 31) == 0 && m) atomicAdd(ctr + idx, (unsigned long long)__popc(m));
}

// dt from the reduced wave speeds: E/sourcecode/euler_timestep.cpp:36-43.
__device__ __forceinline__ double choose_dt(const DevState& s, double maxu, double maxv) {
    double cfl = s.cfl;
    if (s.n < 5) cfl = smin(cfl, 0.2);
    double dt = cfl * smin(s.dx / maxu, s.dy / maxv);
    if (s.t + dt > s.T) dt = s.T - s.t;
    return dt;
}

// Last-CTA finish of the wave-speed reduction.  Partials are combined in CTA
// order, so the mass sums are reproducible run to run.
__device__ inline void finish_reduction(DevState* st, const double* partials, int nblocks,
                                 int advance_time, double dt_used, int flip_cur) {
    __shared__ double red[4][32];
    double mu = 0.0, mv = 0.0, m1 = 0.0, m2 = 0.0;
    // fixed assignment of partials to threads, then a fixed-order tree
    for (int b = threadIdx.x; b < nblocks; b += blockDim.x) {
        mu = smax(mu, partials[4 * b + 0]);
        mv = smax(mv, partials[4 * b + 1]);
        m1 += partials[4 * b + 2];
        m2 += partials[4 * b + 3];
    }
    for (int o = 16; o > 0; o >>= 1) {
        mu = smax(mu, __shfl_down_sync(0xffffffffu, mu, o));
        mv = smax(mv, __shfl_down_sync(0xffffffffu, mv, o));
        m1 += __shfl_down_sync(0xffffffffu, m1, o);
        m2 += __shfl_down_sync(0xffffffffu, m2, o);
    }
    int w = threadIdx.x >> 5, nw = blockDim.x >> 5;
    if ((threadIdx.x & 31) == 0) {
        red[0][w] = mu;
        red[1][w] = mv;
        red[2][w] = m1;
        red[3][w] = m2;
    }
    __syncthreads();
    if (threadIdx.x == 0) {
        mu = red[0][0];
        mv = red[1][0];
        m1 = red[2][0];
        m2 = red[3][0];
        for (int i = 1; i < nw; ++i) {
            mu = smax(mu, red[0][i]);
            mv = smax(mv, red[1][i]);
            m1 += red[2][i];
            m2 += red[3][i];
        }
        DevState s = *st;
        if (advance_time) {
            s.t = s.t + dt_used;
            s.n = s.n + 1;
            if (fabs(s.t - s.T) < 1e-12) s.t = s.T;
        }
        s.maxu = mu;
        s.maxv = mv;
        s.mass1 = m1 * s.dx * s.dy;
        s.mass2 = m2 * s.dx * s.dy;
        s.dt = choose_dt(s, mu, mv);
        s.done = !(s.t < s.T);
        s.ticket = 0;
        if (flip_cur) s.cur ^= 1;
        *st = s;
        __threadfence();
    }
}

// Wave speeds of one stored (unrotated) state, exactly as compute_dt forms
// them.  Returns |u|+c, |v|+c and the mass contributions.
template <int MODEL>
__device__ __forceinline__ void wave_speeds(const Eos& q, const double* U, double& su, double& sv,
                                            double& m1, double& m2) {
    Prim<MODEL> P;
    cons_to_prim<MODEL>(q, U, P);
    double c;
    if constexpr (MODEL == MODEL_EULER) {
        c = sg_soundspeed(q, P.W[3], P.rho);
        m1 = P.rho;
        m2 = 0.0;
    } else {
        c = mix_soundspeed(P.mix, P.rho, P.W[4]);
        m1 = U[0];
        m2 = U[1];
    }
    su = fabs(P.W[ModelTraits<MODEL>::IM]) + c;
    sv = fabs(P.W[ModelTraits<MODEL>::IT]) + c;
}

template <int MODEL, int DIR, int TS, int NA>
struct SweepTile {
    static constexpr int NV = ModelTraits<MODEL>::NV;
    static constexpr int LA = TS + 4;           // staged cells per line
    static constexpr int NSLOT = LA * NA;
    static constexpr int STRIDE = (DIR == DIR_X) ? 1 : NA;  // next cell along the sweep
    // slot of (along a, across b), x fastest in both directions
    __device__ static __forceinline__ int slot(int a, int b) {
        return (DIR == DIR_X) ? b * LA + a : a * NA + b;
    }
    // i-th item of a phase covering along-indices [a0, a0+cnt) on all lines
    __device__ static __forceinline__ void item(int i, int a0, int cnt, int& a, int& b) {
        if (DIR == DIR_X) {
            b = i / cnt;
            a = a0 + i - b * cnt;
        } else {
            a = a0 + i / NA;
            b = i - (i / NA) * NA;
        }
    }
};

struct SweepSmemLayout {
    // offsets in doubles
    int U, WF, EP, EM, FLAGS_BYTES;
};

template <int MODEL, int DIR, int TS, int NA>
__host__ __device__ constexpr int sweep_smem_bytes() {
    using T = SweepTile<MODEL, DIR, TS, NA>;
    // U, W/F (flux needs NV + 2 per face), E+, E-, flags
    return (T::NV * T::NSLOT + (T::NV + 2) * T::NSLOT + 2 * T::NV * T::NSLOT) * 8 + T::NSLOT * 4 +
           4 * 32 * 8;
}

// Bounded for 4 (Euler, 64 registers) and 3 (Allaire, 80 registers) CTAs
// per SM, spilling some 30-40 bytes per thread: 6 % and 7 % faster than at
// 3 and 2 CTAs.
template <int MODEL, int DIR, int TS, int NA>
__global__ void __launch_bounds__(256, MODEL == MODEL_EULER ? 4 : 3) sweep_kernel(SweepArgs A) {
    using Tl = SweepTile<MODEL, DIR, TS, NA>;
    using MT = ModelTraits<MODEL>;
    constexpr int NV = MT::NV;
    constexpr int LA = Tl::LA;
    constexpr int NSLOT = Tl::NSLOT;
    constexpr int ST = Tl::STRIDE;

    extern __shared__ __align__(16) double smem[];
    double* sU = smem;                    // [NV][NSLOT] conserved (rotated in y)
    double* sWF = sU + NV * NSLOT;        // [NV][NSLOT] primitives, later [NV+2][NSLOT] fluxes
    double* sEP = sWF + (NV + 2) * NSLOT; // [NV][NSLOT] state at the cell's high face
    double* sEM = sEP + NV * NSLOT;       // [NV][NSLOT] state at the cell's low face
    unsigned char* sFl = reinterpret_cast<unsigned char*>(sEM + NV * NSLOT);  // flags

    const DevState* st = A.st;
    if (!A.use_host_dt && st->done) return;
    const int cur = st->cur;
    const double* __restrict__ gin = A.bufs[cur ^ A.in_sel];
    double* __restrict__ gout = A.bufs[cur ^ A.in_sel ^ 1];
    const double dt_step = A.use_host_dt ? A.dt_host : st->dt;  // dt of the whole step
    const double dt = A.dt_scale * dt_step;                        // this sweep's dt
    const Eos q = A.eos;
    const int len = (DIR == DIR_X) ? A.nx : A.ny;   // cells along the sweep
    const int wid = (DIR == DIR_X) ? A.ny : A.nx;   // lines
    const int tiles_along = (len + TS - 1) / TS;
    const int t_al = blockIdx.x % tiles_along;
    const int t_ac = blockIdx.x / tiles_along;
    const int a_org = t_al * TS - 2;  // global along-coordinate of staged cell 0
    const int b_org = t_ac * NA;
    const int tid = threadIdx.x;
    constexpr int NT = 256;

    // ---- P1: load (with the boundary ghost fill), rotate, convert --------
    // Ghost cell g (g = -1, -2 or len, len+1) mirrors interior cell -g-1 or
    // 2*len-1-g; a reflective wall negates the normal momentum
    // (E/sourcecode/euler_ppsweep.cpp:16,27).  The y-sweep works on the
    // rotated state (u,v) -> (v,-u) (E/sourcecode/euler_colsweep.cpp:22-29).
    bool bad_in = false;
    for (int i = tid; i < NSLOT; i += NT) {
        int a, b;
        Tl::item(i, 0, LA, a, b);
        int ga = a_org + a, gb = b_org + b;
        bool line_ok = gb < wid;
        int src = ga;
        bool neg = false;
        if (ga < 0) { src = -ga - 1; neg = A.bc_lo; }
        else if (ga >= len) { src = 2 * len - 1 - ga; neg = A.bc_hi; }
        // clamp staged cells beyond the last ghost (partial tiles) into range
        src = min(max(src, 0), len - 1);
        int gbs = line_ok ? gb : wid - 1;
        long long off = (DIR == DIR_X) ? (long long)gbs * A.pitch + src
                                       : (long long)src * A.pitch + gbs;
        double U[NV];
#pragma unroll
        for (int k = 0; k < NV; ++k) U[k] = __ldg(gin + k * A.plane + off);
        if (DIR == DIR_X) {
            if (neg) U[MT::IM] = -U[MT::IM];
        } else {
            if (neg) U[MT::IT] = -U[MT::IT];
            double t = U[MT::IM];
            U[MT::IM] = U[MT::IT];
            U[MT::IT] = -t;
        }
        int s = Tl::slot(a, b);
#pragma unroll
        for (int k = 0; k < NV; ++k) sU[k * NSLOT + s] = U[k];
        Prim<MODEL> P;
        cons_to_prim<MODEL>(q, U, P);
#pragma unroll
        for (int k = 0; k < NV; ++k) sWF[k * NSLOT + s] = P.W[k];
        // reference assert on the stencil states (interior staged cells only)
        bool phys;
        if constexpr (MODEL == MODEL_EULER) phys = P.rho >= 0.0 && P.e >= 0.0;
        else phys = is_physical_exact<MODEL>(U);
        bad_in |= line_ok && ga >= 0 && ga < len && a >= 2 && a < TS + 2 && !phys;
    }
    block_count(A.counters, CNT_UNPHYSICAL_INPUT, bad_in);
    __syncthreads();

    const double s_half = 0.5 * (dt / A.h_flux);
    const double k_upd = dt / A.h_upd;

    // ---- P2: slopes and face states per cell (along 1 .. LA-2) ----------
    if (!A.godunov) {
        for (int i = tid; i < (LA - 2) * NA; i += NT) {
            int a, b;
            Tl::item(i, 1, LA - 2, a, b);
            int s = Tl::slot(a, b);
            Prim<MODEL> P;
            double Wl[NV], Wr[NV], d[NV];
#pragma unroll
            for (int k = 0; k < NV; ++k) {
                P.W[k] = sWF[k * NSLOT + s];
                Wl[k] = sWF[k * NSLOT + s - ST];
                Wr[k] = sWF[k * NSLOT + s + ST];
            }
            limit_all1<NV>(A.limiter, Wl, P.W, Wr, d);
            if constexpr (MODEL == MODEL_EULER) {
                P.rho = P.W[0];
            } else {
                P.rho = P.W[0] + P.W[1];
                P.mix = mix_coeffs(q, P.W[5]);
            }
            // slope-extrapolated states (check only)
            double Wt[NV], Ut[NV], e;
            unsigned fl = 0;
#pragma unroll
            for (int k = 0; k < NV; ++k) Wt[k] = P.W[k] + 0.5 * d[k];
            prim_to_cons<MODEL>(q, Wt, Ut, e);
            if (muscl_check<MODEL>(Ut, Wt, e)) fl |= 1u;  // high face ok
#pragma unroll
            for (int k = 0; k < NV; ++k) Wt[k] = P.W[k] - 0.5 * d[k];
            prim_to_cons<MODEL>(q, Wt, Ut, e);
            if (muscl_check<MODEL>(Ut, Wt, e)) fl |= 2u;  // low face ok
            // half-step evolved states
            double X[NV];
            jacobian_times<MODEL>(q, P, d, s_half, X);
#pragma unroll
            for (int k = 0; k < NV; ++k) Wt[k] = (P.W[k] + 0.5 * d[k]) - X[k];
            prim_to_cons<MODEL>(q, Wt, Ut, e);
            if (muscl_check<MODEL>(Ut, Wt, e)) fl |= 4u;
#pragma unroll
            for (int k = 0; k < NV; ++k) sEP[k * NSLOT + s] = Ut[k];
#pragma unroll
            for (int k = 0; k < NV; ++k) Wt[k] = (P.W[k] - 0.5 * d[k]) - X[k];
            prim_to_cons<MODEL>(q, Wt, Ut, e);
            if (muscl_check<MODEL>(Ut, Wt, e)) fl |= 8u;
#pragma unroll
            for (int k = 0; k < NV; ++k) sEM[k * NSLOT + s] = Ut[k];
            sFl[s] = (unsigned char)fl;
        }
    }
    __syncthreads();

    // ---- P3: flux at each face (along 2 .. TS+2; face a is between a-1, a)
    // The primitive planes are dead after P2, so the fluxes overwrite them;
    // P3 itself reads only sU, sEP, sEM and the flags.
    double* sF = sWF;  // [NV + 2][NSLOT]: flux, u*, z*
    bool ev_zero = false, ev_first = false;
    for (int i = tid; i < (TS + 1) * NA; i += NT) {
        int a, b;
        Tl::item(i, 2, TS + 1, a, b);
        int sR = Tl::slot(a, b), sL = sR - ST;
        double EL[NV], ER[NV];
        bool counted = (b_org + b) < wid && (a_org + a) <= len &&
                       (a < TS + 2 || a_org + a == len);
        if (A.godunov) {
#pragma unroll
            for (int k = 0; k < NV; ++k) {
                EL[k] = sU[k * NSLOT + sL];
                ER[k] = sU[k * NSLOT + sR];
            }
        } else {
            unsigned fL = sFl[sL], fR = sFl[sR];
            bool ok2;
            if ((fL & 1u) && (fR & 2u)) {
#pragma unroll
                for (int k = 0; k < NV; ++k) {
                    EL[k] = sEP[k * NSLOT + sL];
                    ER[k] = sEM[k * NSLOT + sR];
                }
                ok2 = (fL & 4u) && (fR & 8u);
            } else {
                // zero slopes for this face (rare)
                ev_zero |= counted;
                double Ua[NV], Ub[NV], Wt[NV], e;
#pragma unroll
                for (int k = 0; k < NV; ++k) {
                    Ua[k] = sU[k * NSLOT + sL];
                    Ub[k] = sU[k * NSLOT + sR];
                }
                Prim<MODEL> PL, PR;
                cons_to_prim<MODEL>(q, Ua, PL);
                cons_to_prim<MODEL>(q, Ub, PR);
                zero_slope_state<MODEL>(q, PL, s_half, true, Wt);
                prim_to_cons<MODEL>(q, Wt, EL, e);
                bool okL = muscl_check<MODEL>(EL, Wt, e);
                zero_slope_state<MODEL>(q, PR, s_half, false, Wt);
                prim_to_cons<MODEL>(q, Wt, ER, e);
                bool okR = muscl_check<MODEL>(ER, Wt, e);
                ok2 = okL && okR;
            }
            if (!ok2) {
                ev_first |= counted;
#pragma unroll
                for (int k = 0; k < NV; ++k) {
                    EL[k] = sU[k * NSLOT + sL];
                    ER[k] = sU[k * NSLOT + sR];
                }
            }
        }
        double Fv[NV], us;
        hllc_flux<MODEL>(q, A.wavespeed, EL, ER, Fv, us);
#pragma unroll
        for (int k = 0; k < NV; ++k) sF[k * NSLOT + sR] = Fv[k];
        sF[NV * NSLOT + sR] = us;
        if constexpr (MODEL == MODEL_ALLAIRE) {
            double cs = copysign(1.0, us);
            double zs;
            if (A.godunov)  // A/headers/flux_solver_godunov.hpp:33-34
                zs = (((1.0 + cs) / 2.0) * EL[5]) + (((1.0 - cs) / 2.0) * ER[5]);
            else  // A/headers/flux_solver_MUSCLhancock.hpp:375
                zs = ((0.5 * (1.0 + cs)) * EL[5]) + ((0.5 * (1.0 - cs)) * ER[5]);
            sF[(NV + 1) * NSLOT + sR] = zs;
        }
    }
    block_count(A.counters, CNT_SLOPE_ZEROED, ev_zero);
    block_count(A.counters, CNT_FIRST_ORDER, ev_first);
    __syncthreads();

    // ---- P4: update, store, reduce (along 2 .. TS+1) ---------------------
    bool ev_fix = false, ev_bad = false;
    double r_mu = 0.0, r_mv = 0.0, r_m1 = 0.0, r_m2 = 0.0;
    for (int i = tid; i < TS * NA; i += NT) {
        int a, b;
        Tl::item(i, 2, TS, a, b);
        int ga = a_org + a, gb = b_org + b;
        if (ga >= len || gb >= wid) continue;
        int s = Tl::slot(a, b);
        double U[NV], N[NV];
#pragma unroll
        for (int k = 0; k < NV; ++k) {
            U[k] = sU[k * NSLOT + s];
            N[k] = U[k] + (k_upd * (sF[k * NSLOT + s] - sF[k * NSLOT + s + ST]));
        }
        if constexpr (MODEL == MODEL_ALLAIRE) {
            N[5] = z_update(A.godunov, k_upd, sU[5 * NSLOT + s - ST], U[5], sU[5 * NSLOT + s + ST],
                            sF[NV * NSLOT + s], sF[NV * NSLOT + s + ST],
                            sF[(NV + 1) * NSLOT + s], sF[(NV + 1) * NSLOT + s + ST], A.z_min);
            bool changed;
            snap_allaire(N, changed);  // live assert(is_physical_state(...))
            ev_bad |= !is_physical_exact<MODEL>(N);
        }
        if (DIR == DIR_Y) {  // rotate back (E/sourcecode/euler_colsweep.cpp:66-73)
            double t = N[MT::IM];
            N[MT::IM] = -N[MT::IT];
            N[MT::IT] = t;
            double t2 = U[MT::IM];  // old state, unrotated, for the fix-up
            U[MT::IM] = -U[MT::IT];
            U[MT::IT] = t2;
        }
        if constexpr (MODEL == MODEL_EULER) {
            // E/sourcecode/euler_rowsweep.cpp:47-82: restore rho or e from the
            // old state when the update produced rho or e <= 0.  A state with
            // rho > 0 and E*rho clearly above |m|^2/2 passes the exact test.
            bool surely = N[0] > 0.0 && N[3] > 0.0 &&
                          (N[3] * N[0]) > (0.5 * ((N[1] * N[1]) + (N[2] * N[2]))) * (1.0 + 1e-13);
            if (!surely && !is_physical_exact<MODEL>(N)) {
                ev_fix = true;
                double rho = N[0];
                double u = N[1] / rho;
                double v = N[2] / rho;
                double e = (N[3] / rho) - (0.5 * ((u * u) + (v * v)));
                double rho_old = U[0];
                double u_old = U[1] / rho_old;
                double v_old = U[2] / rho_old;
                double e_old = (U[3] / rho_old) - (0.5 * ((u_old * u_old) + (v_old * v_old)));
                if (rho <= 1e-12) rho = rho_old;
                if (e <= 1e-12) e = e_old;
                double W[4] = {rho, u, v, sg_pressure(q, e, rho)};
                double ee;
                prim_to_cons<MODEL>(q, W, N, ee);
            }
        }
        long long off = (DIR == DIR_X) ? (long long)gb * A.pitch + ga : (long long)ga * A.pitch + gb;
#pragma unroll
        for (int k = 0; k < NV; ++k) gout[k * A.plane + off] = N[k];
        if (A.reduce) {
            double su, sv, m1, m2;
            wave_speeds<MODEL>(q, N, su, sv, m1, m2);
            r_mu = smax(r_mu, su);
            r_mv = smax(r_mv, sv);
            r_m1 += m1;
            r_m2 += m2;
        }
    }
    block_count(A.counters, CNT_FIXUP, ev_fix);
    block_count(A.counters, CNT_UNPHYSICAL_OUTPUT, ev_bad);
    if (!A.reduce) return;

    // ---- block reduction, last-CTA finish ---------------------------------
    __shared__ double red[4][8];
    __shared__ bool is_last;
    for (int o = 16; o > 0; o >>= 1) {
        r_mu = smax(r_mu, __shfl_down_sync(0xffffffffu, r_mu, o));
        r_mv = smax(r_mv, __shfl_down_sync(0xffffffffu, r_mv, o));
        r_m1 += __shfl_down_sync(0xffffffffu, r_m1, o);
        r_m2 += __shfl_down_sync(0xffffffffu, r_m2, o);
    }
    if ((tid & 31) == 0) {
        red[0][tid >> 5] = r_mu;
        red[1][tid >> 5] = r_mv;
        red[2][tid >> 5] = r_m1;
        red[3][tid >> 5] = r_m2;
    }
    __syncthreads();
    if (tid == 0) {
        double mu = red[0][0], mv = red[1][0], m1 = red[2][0], m2 = red[3][0];
        for (int w = 1; w < NT / 32; ++w) {
            mu = smax(mu, red[0][w]);
            mv = smax(mv, red[1][w]);
            m1 += red[2][w];
            m2 += red[3][w];
        }
        double* p = A.partials + 4 * blockIdx.x;
        p[0] = mu;
        p[1] = mv;
        p[2] = m1;
        p[3] = m2;
        __threadfence();
        unsigned t = atomicAdd(&A.st->ticket, 1u);
        is_last = (t == gridDim.x - 1);
    }
    __syncthreads();
    if (is_last) {
        __threadfence();
        finish_reduction(A.st, A.partials, gridDim.x, A.advance_time, dt_step, A.flip_cur);
    }
}

}  // namespace cfd
