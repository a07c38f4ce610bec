// Mixed-precision split sweeps over a batch of independent solves.
//
// Same numerical method as the plain FP64 path (cfd_physics.cuh and
// cfd_sweep.cuh, which cite the reference) with this precision split:
//   * state: every conserved component stored as an FP32 value plus an FP32
//     compensation word (hi + lo, kept normalised by an error-free sum), so
//     small increments are not lost to FP32 rounding step after step;
//   * reconstruction, slope limiting, the half step and the HLLC solve in
//     FP32 with hardware reciprocal / square-root approximations;
//   * FP64 for the stiffened-gas pressure recovery p = rho e / eps - k of
//     cells with pinf != 0 (pinf up to 6e8 cancels catastrophically in FP32),
//     for the CFL wave-speed reduction and dt, and for the time accumulator.
// The face states go to the Riemann solver as primitives, so the pressure
// is never re-derived from a reconstructed FP32 energy.
//
// Batching: one launch sweeps every tile of every active instance.  A tile
// table maps blockIdx to (instance, tile); each instance has its own grid,
// materials, options, buffers and device-resident time state, and its y
// sweep finishes its own wave-speed reduction (last CTA of that instance).
#pragma once

#include "cfd_physics.cuh"
#include "cfd_sweep.cuh"

namespace cfd {
namespace mixed {

// Per-instance descriptor (device memory, one per solve).
struct Inst {
    float* hi[2];   // two state buffers, nv planes each
    float* lo[2];
    long long plane;
    int pitch, nx, ny, nv;
    int model, limiter, wavespeed, godunov, fix_dy;
    int bc[4];       // L, R, B, T
    double dx, dy;
    double z_min;
    Eos eos;         // FP64 material parameters
    float g1f, p1f, g2f, p2f, gm1_1f, gm1_2f, gp1f;
    DevState* st;
    double* partials;   // 4 per y tile
    int tiles_x, tiles_y;   // tiles of each sweep
    int max_steps;          // stop after this many steps (and at t >= T)
    int active;             // 0: skip
};

struct MixedArgs {
    Inst* insts;
    const int* tile_inst;   // instance of each tile of this launch
    const int* tile_local;  // tile index within its instance
    int ntiles;             // tiles of this launch; CTAs loop over them (persistent)
};

// This translation unit is compiled with -prec-div=false -prec-sqrt=false:
// single-precision division, reciprocal and square root use the hardware
// approximations (about 1-2 ulp), ample for the FP32 face arithmetic.
__device__ __forceinline__ float frcp(float x) { return 1.0f / x; }
__device__ __forceinline__ float fdiv(float a, float b) { return a / b; }
__device__ __forceinline__ float fsqrt(float x) { return sqrtf(x); }
__device__ __forceinline__ float fminf_s(float a, float b) { return (b < a) ? b : a; }
__device__ __forceinline__ float fmaxf_s(float a, float b) { return (a < b) ? b : a; }

// Mixture coefficients eps(z), k(z) in FP32 and FP64.
__device__ __forceinline__ void mix_f(const Inst& I, float z, float& eps, float& k) {
    float omz = 1.0f - z;
    eps = fdiv(z, I.gm1_1f) + fdiv(omz, I.gm1_2f);
    float num = fdiv(z * I.g1f * I.p1f, I.gm1_1f) + fdiv(omz * I.g2f * I.p2f, I.gm1_2f);
    k = fdiv(num, eps);
}

// Primitive state (rho-split for Allaire: W = rho1 z, rho2 (1-z), u, v, p, z).
template <int MODEL> struct PrimF {
    float W[ModelTraits<MODEL>::NV];
};

// Conserved (hi + lo) -> primitive.  The pressure of a stiffened gas comes
// from the FP64 sum hi + lo.
template <int MODEL>
__device__ __forceinline__ void c2p_mixed(const Inst& I, const float* hi, const float* lo,
                                          float* W) {
    if constexpr (MODEL == MODEL_EULER) {
        float rho = hi[0];
        float r = frcp(rho);
        float u = hi[1] * r, v = hi[2] * r;
        float p;
        if (I.p1f == 0.0f) {
            p = I.gm1_1f * (hi[3] - 0.5f * (hi[1] * u + hi[2] * v));
        } else {
            double R = (double)hi[0] + (double)lo[0];
            double M1 = (double)hi[1] + (double)lo[1], M2 = (double)hi[2] + (double)lo[2];
            double E = (double)hi[3] + (double)lo[3];
            double re = E - 0.5 * (M1 * M1 + M2 * M2) / R;
            p = (float)(I.eos.gm1_1 * re - I.eos.gp1);
        }
        W[0] = rho;
        W[1] = u;
        W[2] = v;
        W[3] = p;
    } else {
        float rho = hi[0] + hi[1];
        float r = frcp(rho);
        float u = hi[2] * r, v = hi[3] * r;
        float z = hi[5];
        float p;
        if (I.p1f == 0.0f && I.p2f == 0.0f) {
            float eps, k;
            mix_f(I, z, eps, k);
            p = fdiv(hi[4] - 0.5f * (hi[2] * u + hi[3] * v), eps);
        } else {
            double R = ((double)hi[0] + (double)lo[0]) + ((double)hi[1] + (double)lo[1]);
            double M1 = (double)hi[2] + (double)lo[2], M2 = (double)hi[3] + (double)lo[3];
            double E = (double)hi[4] + (double)lo[4];
            double zz = (double)hi[5] + (double)lo[5];
            Mix m = mix_coeffs(I.eos, zz);
            double re = E - 0.5 * (M1 * M1 + M2 * M2) / R;
            p = (float)(re / m.eps - m.k);
        }
        W[0] = hi[0];
        W[1] = hi[1];
        W[2] = u;
        W[3] = v;
        W[4] = p;
        W[5] = z;
    }
}

// Physical primitive state: the conversion to conserved variables would give
// rho >= 0 and e >= 0 (and 0 <= z <= 1, partial densities >= 0).
template <int MODEL> __device__ __forceinline__ bool phys_prim(const Inst& I, const float* W) {
    if constexpr (MODEL == MODEL_EULER) {
        return W[0] >= 0.0f && W[3] + I.gp1f >= 0.0f;
    } else {
        float eps, k;
        mix_f(I, W[5], eps, k);
        return W[0] >= 0.0f && W[1] >= 0.0f && W[5] >= 0.0f && W[5] <= 1.0f && W[4] + k >= 0.0f;
    }
}

__device__ __forceinline__ float limit_f(int lim, float a, float b) {
    switch (lim) {
        case LIM_VANLEER:
            return (a * b > 0.0f) ? fdiv(2.0f * a * b, a + b) : 0.0f;
        case LIM_MC:
            if (b >= 0.0f && a >= 0.0f) return fminf_s(0.5f * (a + b), fminf_s(2.0f * a, 2.0f * b));
            if (b <= 0.0f && a <= 0.0f) return fmaxf_s(0.5f * (a + b), fmaxf_s(2.0f * a, 2.0f * b));
            return 0.0f;
        case LIM_UNLIMITED:
            return 0.5f * (a + b);
        default:
            return (b > 0.0f) ? fmaxf_s(0.0f, fminf_s(a, b)) : fminf_s(0.0f, fmaxf_s(a, b));
    }
}

// Sound speed of a primitive state.
template <int MODEL> __device__ __forceinline__ float sound_f(const Inst& I, const float* W) {
    if constexpr (MODEL == MODEL_EULER) {
        return fsqrt(fmaxf_s(0.0f, fdiv(I.g1f * (W[3] + I.p1f), W[0])));
    } else {
        float eps, k;
        mix_f(I, W[5], eps, k);
        float rho = W[0] + W[1];
        return fsqrt(fmaxf_s(0.0f, fdiv(k + W[4] * (frcp(eps) + 1.0f), rho)));
    }
}

// Half-step evolution X = (0.5 dt/dx) A(W) d (primitive Jacobian).
template <int MODEL>
__device__ __forceinline__ void jac_f(const Inst& I, const float* W, const float* d, float s,
                                      float* X) {
    float c = sound_f<MODEL>(I, W);
    if constexpr (MODEL == MODEL_EULER) {
        float rho = W[0], u = W[1];
        X[0] = s * (u * d[0] + rho * d[1]);
        X[1] = s * (u * d[1] + frcp(rho) * d[3]);
        X[2] = s * (u * d[2]);
        X[3] = s * (rho * c * c * d[1] + u * d[3]);
    } else {
        float rho = W[0] + W[1], u = W[2];
        X[0] = s * (u * d[0] + W[0] * d[2]);
        X[1] = s * (u * d[1] + W[1] * d[2]);
        X[2] = s * (u * d[2] + frcp(rho) * d[4]);
        X[3] = s * (u * d[3]);
        X[4] = s * (rho * c * c * d[2] + u * d[4]);
        X[5] = s * (u * d[5]);
    }
}

// HLLC flux from primitive face states (same wave-speed estimates and star
// states as hllc_flux in cfd_physics.cuh).  F[NV] = flux, F[NV] = u*,
// F[NV+1] = z* (Allaire).
template <int MODEL>
__device__ __forceinline__ void hllc_prim(const Inst& I, const float* WL, const float* WR,
                                          float* F) {
    using T = ModelTraits<MODEL>;
    constexpr int NV = T::NV;
    float rL, rR, uL, uR, pL, pR, cL, cR, epsL = 1.f, kL = 0.f, epsR = 1.f, kR = 0.f;
    if constexpr (MODEL == MODEL_EULER) {
        rL = WL[0]; uL = WL[1]; pL = WL[3];
        rR = WR[0]; uR = WR[1]; pR = WR[3];
        cL = fsqrt(fmaxf_s(0.0f, fdiv(I.g1f * (pL + I.p1f), rL)));
        cR = fsqrt(fmaxf_s(0.0f, fdiv(I.g1f * (pR + I.p1f), rR)));
    } else {
        rL = WL[0] + WL[1]; uL = WL[2]; pL = WL[4];
        rR = WR[0] + WR[1]; uR = WR[2]; pR = WR[4];
        mix_f(I, WL[5], epsL, kL);
        mix_f(I, WR[5], epsR, kR);
        cL = fsqrt(fmaxf_s(0.0f, fdiv(kL + pL * (frcp(epsL) + 1.0f), rL)));
        cR = fsqrt(fmaxf_s(0.0f, fdiv(kR + pR * (frcp(epsR) + 1.0f), rR)));
    }
    float SL, SR;
    if (MODEL == MODEL_ALLAIRE && I.wavespeed == WS_PVRS) {
        float ra = 0.5f * (rL + rR), ca = 0.5f * (cL + cR);
        float ppv = fmaxf_s(0.0f, 0.5f * (pL + pR) + 0.5f * (uL - uR) * ra * ca);
        if (ppv > pL) {
            float pa = 0.5f * (ppv + pL);
            SL = uL - fsqrt(fmaxf_s(0.0f, fdiv(ppv + kL + fdiv(pa, epsL), rL)));
        } else {
            SL = uL - cL;
        }
        if (ppv > pR) {
            float pa = 0.5f * (ppv + pR);
            SR = uR + fsqrt(fmaxf_s(0.0f, fdiv(ppv + kR + fdiv(pa, epsR), rR)));
        } else {
            SR = uR + cR;
        }
    } else {
        float ua = 0.5f * (uL + uR), ca = 0.5f * (cL + cR);
        SL = fminf_s(ua - ca, uL - cL);
        SR = fmaxf_s(ua + ca, uR + cR);
    }
    float dSL = SL - uL, dSR = SR - uR;
    float us = fdiv((pR - pL) + rL * uL * dSL - rR * uR * dSR, rL * dSL - rR * dSR);
    bool left = !signbit(us);
    const float* W = left ? WL : WR;
    float rho = left ? rL : rR, u = left ? uL : uR, p = left ? pL : pR;
    float Sk = left ? SL : SR, dS = left ? dSL : dSR;
    float wave = left ? fminf_s(0.0f, SL) : fmaxf_s(0.0f, SR);
    float fac = fdiv(dS, Sk - us);
    // conserved state of the selected side
    float U[NV];
    if constexpr (MODEL == MODEL_EULER) {
        float v = W[2];
        U[0] = rho;
        U[1] = rho * u;
        U[2] = rho * v;
        U[3] = fdiv(p + I.gp1f, I.gm1_1f) + 0.5f * rho * (u * u + v * v);
    } else {
        float v = W[3];
        float eps = left ? epsL : epsR, k = left ? kL : kR;
        U[0] = W[0];
        U[1] = W[1];
        U[2] = rho * u;
        U[3] = rho * v;
        U[4] = (p + k) * eps + 0.5f * rho * (u * u + v * v);
        U[5] = W[5];
    }
    float Us[NV];
#pragma unroll
    for (int k = 0; k < NV; ++k) Us[k] = fac * U[k];
    Us[T::IM] = fac * rho * us;
    Us[T::IE] = fac * (U[T::IE] + (us - u) * (rho * us + fdiv(p, dS)));
    float Fp[NV];
    if constexpr (MODEL == MODEL_EULER) {
        Fp[0] = U[0] * u;
        Fp[1] = U[1] * u + p;
        Fp[2] = U[2] * u;
        Fp[3] = (U[3] + p) * u;
    } else {
        Fp[0] = U[0] * u;
        Fp[1] = U[1] * u;
        Fp[2] = U[2] * u + p;
        Fp[3] = U[3] * u;
        Fp[4] = (U[4] + p) * u;
        Fp[5] = 0.0f;
        Us[5] = U[5];
    }
#pragma unroll
    for (int k = 0; k < NV; ++k) F[k] = Fp[k] + wave * (Us[k] - U[k]);
    if constexpr (MODEL == MODEL_ALLAIRE) F[5] = 0.0f;
    F[NV] = us;
    if constexpr (MODEL == MODEL_ALLAIRE) F[NV + 1] = left ? WL[5] : WR[5];
}

// hi + lo += d with an error-free transformation (TwoSum), keeping the pair
// normalised.
__device__ __forceinline__ void comp_add(float& hi, float& lo, float d) {
    float y = lo + d;
    float s = hi + y;
    float bp = s - hi;
    float e = (hi - (s - bp)) + (y - bp);
    hi = s;
    lo = e;
}

template <int MODEL, int DIR, int TS, int NA>
struct MTile {
    static constexpr int NV = ModelTraits<MODEL>::NV;
    static constexpr int LA = TS + 4;
    static constexpr int NSLOT = LA * NA;
    static constexpr int ST = (DIR == DIR_X) ? 1 : NA;
    __device__ static __forceinline__ int slot(int a, int b) {
        return (DIR == DIR_X) ? b * LA + a : a * NA + b;
    }
    __device__ static __forceinline__ void item(int i, int a0, int cnt, int& a, int& b) {
        if (DIR == DIR_X) {
            b = i / cnt;
            a = a0 + i - b * cnt;
        } else {
            a = a0 + i / NA;
            b = i - (i / NA) * NA;
        }
    }
    // floats: hi, lo, W (NV each), Wp, Wm (NV each), F (NV + 2); bytes: flags
    static constexpr int SMEM = (6 * NV + 2) * NSLOT * 4 + NSLOT + 64;
};

template <int MODEL, int DIR, int TS, int NA>
__device__ __forceinline__ void mixed_tile(const MixedArgs& A, int tile, float* fsm) {
    using Tl = MTile<MODEL, DIR, TS, NA>;
    using MT = ModelTraits<MODEL>;
    constexpr int NV = MT::NV, LA = Tl::LA, NSLOT = Tl::NSLOT, ST = Tl::ST, NT = 256;
    float* sHi = fsm;
    float* sLo = sHi + NV * NSLOT;
    float* sW = sLo + NV * NSLOT;
    float* sWp = sW + NV * NSLOT;
    float* sWm = sWp + NV * NSLOT;
    float* sF = sWm + NV * NSLOT;  // NV + 2 planes
    unsigned char* sFl = reinterpret_cast<unsigned char*>(sF + (NV + 2) * NSLOT);

    const int inst = A.tile_inst[tile];
    const int ltile = A.tile_local[tile];
    const Inst& I = A.insts[inst];
    DevState* st = I.st;
    if (!I.active || st->done || st->n >= I.max_steps) return;
    const int cur = st->cur;
    const float* __restrict__ ghi = I.hi[cur ^ (DIR == DIR_Y)];
    const float* __restrict__ glo = I.lo[cur ^ (DIR == DIR_Y)];
    float* __restrict__ ohi = I.hi[cur ^ (DIR == DIR_X)];
    float* __restrict__ olo = I.lo[cur ^ (DIR == DIR_X)];
    const double dt = st->dt;
    const int len = (DIR == DIR_X) ? I.nx : I.ny;
    const int wid = (DIR == DIR_X) ? I.ny : I.nx;
    const int tiles_along = (len + TS - 1) / TS;
    const int a_org = (ltile % tiles_along) * TS - 2;
    const int b_org = (ltile / tiles_along) * NA;
    const int bc_lo = (DIR == DIR_X) ? I.bc[0] : I.bc[2];
    const int bc_hi = (DIR == DIR_X) ? I.bc[1] : I.bc[3];
    const int tid = threadIdx.x;
    const double h_flux = (DIR == DIR_X) ? I.dx : (I.fix_dy ? I.dy : I.dx);
    const double h_upd = (DIR == DIR_X) ? I.dx : I.dy;
    const float s_half = (float)(0.5 * (dt / h_flux));
    const float k_upd = (float)(dt / h_upd);

    // ---- P1: load hi/lo with the boundary fill, rotate, convert --------
    for (int i = tid; i < NSLOT; i += NT) {
        int a, b;
        Tl::item(i, 0, LA, a, b);
        int ga = a_org + a, gb = b_org + b;
        int src = ga;
        bool neg = false;
        if (ga < 0) { src = -ga - 1; neg = bc_lo; }
        else if (ga >= len) { src = 2 * len - 1 - ga; neg = bc_hi; }
        src = min(max(src, 0), len - 1);
        int gbs = min(gb, wid - 1);
        long long off = (DIR == DIR_X) ? (long long)gbs * I.pitch + src : (long long)src * I.pitch + gbs;
        float h[NV], l[NV];
#pragma unroll
        for (int k = 0; k < NV; ++k) {
            h[k] = __ldg(ghi + k * I.plane + off);
            l[k] = __ldg(glo + k * I.plane + off);
        }
        if (DIR == DIR_X) {
            if (neg) { h[MT::IM] = -h[MT::IM]; l[MT::IM] = -l[MT::IM]; }
        } else {
            if (neg) { h[MT::IT] = -h[MT::IT]; l[MT::IT] = -l[MT::IT]; }
            float t = h[MT::IM], tl = l[MT::IM];
            h[MT::IM] = h[MT::IT]; l[MT::IM] = l[MT::IT];
            h[MT::IT] = -t; l[MT::IT] = -tl;
        }
        int s = Tl::slot(a, b);
        float W[NV];
        c2p_mixed<MODEL>(I, h, l, W);
#pragma unroll
        for (int k = 0; k < NV; ++k) {
            sHi[k * NSLOT + s] = h[k];
            sLo[k * NSLOT + s] = l[k];
            sW[k * NSLOT + s] = W[k];
        }
    }
    __syncthreads();

    // ---- P2: slopes and evolved face states (primitive) ----------------
    if (!I.godunov) {
        for (int i = tid; i < (LA - 2) * NA; i += NT) {
            int a, b;
            Tl::item(i, 1, LA - 2, a, b);
            int s = Tl::slot(a, b);
            float W[NV], d[NV], X[NV], Wt[NV];
#pragma unroll
            for (int k = 0; k < NV; ++k) {
                W[k] = sW[k * NSLOT + s];
                d[k] = limit_f(I.limiter, W[k] - sW[k * NSLOT + s - ST], sW[k * NSLOT + s + ST] - W[k]);
            }
            unsigned fl = 0;
#pragma unroll
            for (int k = 0; k < NV; ++k) Wt[k] = W[k] + 0.5f * d[k];
            if (phys_prim<MODEL>(I, Wt)) fl |= 1u;
#pragma unroll
            for (int k = 0; k < NV; ++k) Wt[k] = W[k] - 0.5f * d[k];
            if (phys_prim<MODEL>(I, Wt)) fl |= 2u;
            jac_f<MODEL>(I, W, d, s_half, X);
#pragma unroll
            for (int k = 0; k < NV; ++k) Wt[k] = (W[k] + 0.5f * d[k]) - X[k];
            if (phys_prim<MODEL>(I, Wt)) fl |= 4u;
#pragma unroll
            for (int k = 0; k < NV; ++k) sWp[k * NSLOT + s] = Wt[k];
#pragma unroll
            for (int k = 0; k < NV; ++k) Wt[k] = (W[k] - 0.5f * d[k]) - X[k];
            if (phys_prim<MODEL>(I, Wt)) fl |= 8u;
#pragma unroll
            for (int k = 0; k < NV; ++k) sWm[k * NSLOT + s] = Wt[k];
            sFl[s] = (unsigned char)fl;
        }
    }
    __syncthreads();

    // ---- P3: HLLC per face -------------------------------------------------
    for (int i = tid; i < (TS + 1) * NA; i += NT) {
        int a, b;
        Tl::item(i, 2, TS + 1, a, b);
        int sR = Tl::slot(a, b), sL = sR - ST;
        float WL[NV], WR[NV];
        bool first = true;
        if (!I.godunov) {
            unsigned fL = sFl[sL], fR = sFl[sR];
            // zero slopes evolve to the cell state itself; the first-order
            // fallback uses the cell states too
            if ((fL & 1u) && (fR & 2u) && (fL & 4u) && (fR & 8u)) {
                first = false;
#pragma unroll
                for (int k = 0; k < NV; ++k) {
                    WL[k] = sWp[k * NSLOT + sL];
                    WR[k] = sWm[k * NSLOT + sR];
                }
            }
        }
        if (first) {
#pragma unroll
            for (int k = 0; k < NV; ++k) {
                WL[k] = sW[k * NSLOT + sL];
                WR[k] = sW[k * NSLOT + sR];
            }
        }
        float F[NV + 2];
        hllc_prim<MODEL>(I, WL, WR, F);
#pragma unroll
        for (int k = 0; k < NV + 2; ++k) sF[k * NSLOT + sR] = F[k];
    }
    __syncthreads();

    // ---- P4: compensated update, store, reduce -----------------------------
    double r_mu = 0.0, r_mv = 0.0, r_m1 = 0.0, r_m2 = 0.0;
    for (int i = tid; i < TS * NA; i += NT) {
        int a, b;
        Tl::item(i, 2, TS, a, b);
        int ga = a_org + a, gb = b_org + b;
        if (ga >= len || gb >= wid) continue;
        int s = Tl::slot(a, b);
        float h[NV], l[NV];
#pragma unroll
        for (int k = 0; k < NV; ++k) {
            h[k] = sHi[k * NSLOT + s];
            l[k] = sLo[k * NSLOT + s];
        }
        float oh[NV], ol[NV];
#pragma unroll
        for (int k = 0; k < NV; ++k) {
            oh[k] = h[k];
            ol[k] = l[k];
        }
#pragma unroll
        for (int k = 0; k < NV; ++k) {
            if (MODEL == MODEL_ALLAIRE && k == 5) continue;
            float dlt = k_upd * (sF[k * NSLOT + s] - sF[k * NSLOT + s + ST]);
            comp_add(h[k], l[k], dlt);
        }
        if constexpr (MODEL == MODEL_ALLAIRE) {
            float usL = sF[NV * NSLOT + s], usR = sF[NV * NSLOT + s + ST];
            float zsL = sF[(NV + 1) * NSLOT + s], zsR = sF[(NV + 1) * NSLOT + s + ST];
            float z = h[5];
            float dz;
            if (I.godunov) {
                float zL = sHi[5 * NSLOT + s - ST], zR = sHi[5 * NSLOT + s + ST];
                dz = -k_upd * ((zR - z) * fminf_s(0.0f, usR) + (z - zL) * fmaxf_s(0.0f, usL));
            } else {
                dz = -k_upd * ((usR * zsR - usL * zsL) - z * (usR - usL));
            }
            comp_add(h[5], l[5], dz);
            float zlo = (float)I.z_min, zhi = (float)(1.0 - I.z_min);
            if (h[5] + l[5] < zlo) { h[5] = zlo; l[5] = (float)(I.z_min - (double)zlo); }
            if (h[5] + l[5] > zhi) { h[5] = zhi; l[5] = (float)((1.0 - I.z_min) - (double)zhi); }
            if (h[0] < 0.0f) { h[0] = 0.0f; l[0] = 0.0f; }
            if (h[1] < 0.0f) { h[1] = 0.0f; l[1] = 0.0f; }
        }
        if (DIR == DIR_Y) {  // rotate back
            float t = h[MT::IM], tl = l[MT::IM];
            h[MT::IM] = -h[MT::IT]; l[MT::IM] = -l[MT::IT];
            h[MT::IT] = t; l[MT::IT] = tl;
            float t2 = oh[MT::IM], t2l = ol[MT::IM];
            oh[MT::IM] = -oh[MT::IT]; ol[MT::IM] = -ol[MT::IT];
            oh[MT::IT] = t2; ol[MT::IT] = t2l;
        }
        float Wn[NV];
        c2p_mixed<MODEL>(I, h, l, Wn);
        if constexpr (MODEL == MODEL_EULER) {
            // density / energy restore as in the plain form (rare)
            if (!(h[0] > 1e-12f) || !(Wn[3] + I.gp1f > 0.0f)) {
                float Wo[NV];
                c2p_mixed<MODEL>(I, oh, ol, Wo);
                float rho = h[0] > 1e-12f ? h[0] : oh[0];
                float u = Wn[1], v = Wn[2];
                float p = (Wn[3] + I.gp1f > 0.0f) ? Wn[3] : Wo[3];
                h[0] = rho; l[0] = 0.f;
                h[1] = rho * u; l[1] = 0.f;
                h[2] = rho * v; l[2] = 0.f;
                h[3] = fdiv(p + I.gp1f, I.gm1_1f) + 0.5f * rho * (u * u + v * v); l[3] = 0.f;
                Wn[0] = rho;
                Wn[3] = p;
            }
        }
        long long off = (DIR == DIR_X) ? (long long)gb * I.pitch + ga : (long long)ga * I.pitch + gb;
#pragma unroll
        for (int k = 0; k < NV; ++k) {
            ohi[k * I.plane + off] = h[k];
            olo[k * I.plane + off] = l[k];
        }
        if (DIR == DIR_Y) {
            float c = sound_f<MODEL>(I, Wn);
            float u = Wn[MT::IM], v = Wn[MT::IT];
            r_mu = smax(r_mu, (double)(fabsf(u) + c));
            r_mv = smax(r_mv, (double)(fabsf(v) + c));
            if constexpr (MODEL == MODEL_EULER) {
                r_m1 += (double)h[0] + (double)l[0];
            } else {
                r_m1 += (double)h[0] + (double)l[0];
                r_m2 += (double)h[1] + (double)l[1];
            }
        }
    }
    if constexpr (DIR == DIR_Y) {

        // ---- per-instance reduction; the instance's last CTA picks its dt ------
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
            double* p = I.partials + 4 * ltile;
            p[0] = mu;
            p[1] = mv;
            p[2] = m1;
            p[3] = m2;
            __threadfence();
            unsigned t = atomicAdd(&st->ticket, 1u);
            is_last = (t == (unsigned)I.tiles_y - 1);
        }
        __syncthreads();
        if (is_last) {
            __threadfence();
            finish_reduction(st, I.partials, I.tiles_y, 1, dt, 0);
        }
    }
}

// Persistent sweep: a fixed grid of CTAs walks the tile list of every
// instance in the launch.
template <int MODEL, int DIR, int TS, int NA>
__global__ void __launch_bounds__(256) mixed_sweep_kernel(MixedArgs A) {
    extern __shared__ __align__(16) float fsm[];
    for (int tile = blockIdx.x; tile < A.ntiles; tile += gridDim.x) {
        mixed_tile<MODEL, DIR, TS, NA>(A, tile, fsm);
        __syncthreads();  // shared memory is reused by the next tile
    }
}

}  // namespace mixed
}  // namespace cfd
