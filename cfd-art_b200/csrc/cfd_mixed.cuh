// Mixed-precision split sweeps over a batch of independent solves.
//
// Same numerical method as the plain FP64 path (cfd_physics.cuh and
// cfd_sweep.cuh, which cite the reference) with this precision split:
//   * state: every conserved component stored as an FP32 value plus an FP32
//     compensation word (hi + lo, kept normalised by an error-free sum), so
//     small increments are not lost to FP32 rounding step after step;
//   * reconstruction, slope limiting, the half step and the HLLC solve in
//     FP32 with hardware reciprocal / square-root approximations;
//   * FP64 for the numerator and denominator of the stiffened-gas pressure
//     p = rho e / eps - k of cells with pinf != 0 (pinf up to 6e8 cancels
//     catastrophically in FP32), for the sums of the CFL reduction, for dt
//     and for the time accumulator.
// The face states go to the Riemann solver as primitives, so the pressure
// is never re-derived from a reconstructed FP32 energy.
//
// Batching: one launch sweeps every tile of every active instance.  A tile
// table maps blockIdx to (instance, tile); each instance has its own grid,
// materials, options, buffers and device-resident time state, and its y
// sweep finishes its own wave-speed reduction (last CTA of that instance).
// The batch's y sweep marches strips by default (cfd_march.cuh) and offers
// this tiled form as three alternative shapes with the same results; the x
// sweep uses the warp segments of cfd_march.cuh.  The tiled code is written
// for both directions, but only its y instantiations are launched.
#pragma once

#include "cfd_physics.cuh"
#include "cfd_sweep.cuh"

namespace cfd {
namespace mixed {

// Per-instance descriptor (device memory, one per solve).  The state of a
// cell is stored packed: components 0-3 as one float4 and, for the Allaire
// model, components 4-5 (E, z) as one float2, each with its compensation
// word in a parallel plane, so a cell is read and written with 2 (Euler) or
// 4 (Allaire) vector accesses.
struct Inst {
    float4* q4[2][2];   // [state buffer][0: value, 1: compensation]
    float2* q2[2][2];   // Allaire only
    long long plane;    // cells per plane (pitch * ny)
    int pitch, nx, ny, nv;
    int model, limiter, wavespeed, godunov, fix_dy;
    int bc[4];       // L, R, B, T
    double dx, dy;
    double z_min;
    Eos eos;         // FP64 material parameters
    // FP32 constants of the sweeps (loaded into registers once per tile):
    // g1, p1, g1 - 1, g1 p1, 1/(g1 - 1), 1/(g2 - 1), g1 p1/(g1 - 1), g2 p2/(g2 - 1)
    alignas(16) float pf[8];
    int flags;       // limiter (bits 0-1), PVRS speeds (2), Godunov (3), stiffened gas (4),
                     // reflective walls L, R, B, T (5-8)
    // FP64 mixture constants for the pressure of stiffened-gas cells:
    // 1/(g1 - 1), 1/(g2 - 1), g1 p1/(g1 - 1), g2 p2/(g2 - 1)
    double pd[4];
    DevState* st;
    double* partials;   // 4 per y tile
    int tiles_x, tiles_y;   // tiles of each sweep
    int max_steps;          // stop after this many steps (and at t >= T)
    int active;             // 0: skip
    int fp64;               // 1: the planes hold FP64 values (fast FP64 form, cfd_fast64.cuh)
};

// One tile of a launch, precomputed on the host when the membership or the
// tile shapes change.
struct alignas(16) TileEnt {
    int inst;          // instance
    int local;         // tile index within the instance
    int a_org, b_org;  // first staged cell along the sweep (halo included), first line
    int len, wid;      // cells along the sweep and lines of the instance
    int max_steps, active;
};

struct MixedArgs {
    Inst* insts;
    const TileEnt* tiles;   // tiles of this launch
    int ntiles;             // tiles of this launch
    int chunk;              // CTA c walks tiles [c * chunk, (c + 1) * chunk) (persistent)
    int rows;               // marching strips: cells along the sweep per strip
};

// Per-tile constants held in registers (one vector load per tile instead of
// a global load at every use).
struct MPar {
    float g1, p1, gm1, gp1, i1, i2, c1, c2;
    int flags;
    __device__ __forceinline__ int limiter() const { return flags & 3; }
    __device__ __forceinline__ bool pvrs() const { return (flags >> 2) & 1; }
    __device__ __forceinline__ bool godunov() const { return (flags >> 3) & 1; }
    __device__ __forceinline__ bool stiff() const { return (flags >> 4) & 1; }
};
enum { MF_PVRS = 4, MF_GODUNOV = 8, MF_STIFF = 16, MF_BC = 32 };  // MF_BC << k: wall on side k (L, R, B, T)

__device__ __forceinline__ MPar load_par(const Inst& I) {
    const float4 a = *reinterpret_cast<const float4*>(I.pf);
    const float4 b = *reinterpret_cast<const float4*>(I.pf + 4);
    MPar P;
    P.g1 = a.x; P.p1 = a.y; P.gm1 = a.z; P.gp1 = a.w;
    P.i1 = b.x; P.i2 = b.y; P.c1 = b.z; P.c2 = b.w;
    P.flags = I.flags;
    return P;
}

// Asynchronous global -> shared copies (no registers held while in flight).
__device__ __forceinline__ void cp_async16(void* smem_dst, const void* gsrc) {
    unsigned sa = (unsigned)__cvta_generic_to_shared(smem_dst);
    asm volatile("cp.async.cg.shared.global [%0], [%1], 16;\n" ::"r"(sa), "l"(gsrc) : "memory");
}
__device__ __forceinline__ void cp_async8(void* smem_dst, const void* gsrc) {
    unsigned sa = (unsigned)__cvta_generic_to_shared(smem_dst);
    asm volatile("cp.async.ca.shared.global [%0], [%1], 8;\n" ::"r"(sa), "l"(gsrc) : "memory");
}
__device__ __forceinline__ void cp_async_commit() { asm volatile("cp.async.commit_group;\n" ::: "memory"); }
__device__ __forceinline__ void cp_async_wait_all() { asm volatile("cp.async.wait_group 0;\n" ::: "memory"); }

__device__ __forceinline__ float frcp(float x) { return 1.0f / x; }
// Approximate quotient without the operand range scaling of `a / b` (which
// only matters for |b| > 2^126; every divisor here, a density, a pressure,
// a wave speed or a product of them, is many orders of magnitude smaller).
// Measured 3-4 % faster on the sweeps, the same results on every test case.
__device__ __forceinline__ float fdiv(float a, float b) { return __fdividef(a, b); }
__device__ __forceinline__ float fsqrt(float x) { return sqrtf(x); }
__device__ __forceinline__ float fminf_s(float a, float b) { return (b < a) ? b : a; }
__device__ __forceinline__ float fmaxf_s(float a, float b) { return (a < b) ? b : a; }

// Mixture coefficients eps(z) = z/(g1-1) + (1-z)/(g2-1) and
// k(z) = (z g1 p1/(g1-1) + (1-z) g2 p2/(g2-1)) / eps in FP32.
__device__ __forceinline__ void mix_f(const MPar& P, float z, float& eps, float& k) {
    float omz = 1.0f - z;
    eps = z * P.i1 + omz * P.i2;
    k = (z * P.c1 + omz * P.c2) * frcp(eps);
}

// Primitive state (rho-split for Allaire: W = rho1 z, rho2 (1-z), u, v, p, z).
template <int MODEL> struct PrimF {
    float W[ModelTraits<MODEL>::NV];
};

// Conserved (hi + lo) -> primitive.  The pressure of a stiffened gas comes
// from the FP64 sum hi + lo.
template <int MODEL>
__device__ __forceinline__ void c2p_mixed(const Inst& I, const MPar& P, const float* hi,
                                          const float* lo, float* W) {
    if constexpr (MODEL == MODEL_EULER) {
        float rho = hi[0];
        float r = frcp(rho);
        float u = hi[1] * r, v = hi[2] * r;
        float p;
        if (!P.stiff()) {
            p = P.gm1 * (hi[3] - 0.5f * (hi[1] * u + hi[2] * v));
        } else {
            double R = (double)hi[0] + (double)lo[0];
            double M1 = (double)hi[1] + (double)lo[1], M2 = (double)hi[2] + (double)lo[2];
            double E = (double)hi[3] + (double)lo[3];
            double re = E - 0.5 * (M1 * M1 + M2 * M2) / R;
            p = (float)(__ldg(&I.eos.gm1_1) * re - __ldg(&I.eos.gp1));
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
        if (!P.stiff()) {
            float eps = z * P.i1 + (1.0f - z) * P.i2;
            p = fdiv(hi[4] - 0.5f * (hi[2] * u + hi[3] * v), eps);
        } else {
            // p = (rho e - kn) / eps with rho e = E - |M|^2 / (2 R) and
            // kn = eps k, as (E R - |M|^2/2 - kn R) / (R eps): numerator and
            // denominator in FP64 (the cancellation of p_inf happens in the
            // numerator), the quotient in FP32, the precision of the result
            double R = ((double)hi[0] + (double)lo[0]) + ((double)hi[1] + (double)lo[1]);
            double M1 = (double)hi[2] + (double)lo[2], M2 = (double)hi[3] + (double)lo[3];
            double E = (double)hi[4] + (double)lo[4];
            double zz = (double)hi[5] + (double)lo[5];
            double omz = 1.0 - zz;
            double eps = zz * __ldg(I.pd + 0) + omz * __ldg(I.pd + 1);
            double kn = zz * __ldg(I.pd + 2) + omz * __ldg(I.pd + 3);
            p = fdiv((float)((E * R - 0.5 * (M1 * M1 + M2 * M2)) - kn * R), (float)(R * eps));
        }
        W[0] = hi[0];
        W[1] = hi[1];
        W[2] = u;
        W[3] = v;
        W[4] = p;
        W[5] = z;
    }
}

// Physical primitive state: the reference's test on the conserved state
// (E/headers/misc_euler.hpp:123-131, A/headers/misc.hpp:228-237) passes,
// i.e. rho >= 0 and e >= 0 (and 0 <= z <= 1, partial densities >= 0).  Its
// e is computed with divisions by rho, so a zero density gives e = NaN and
// fails the test: the density must be strictly positive (a face state of
// zero density taken as physical produced infinite sound speeds and NaN
// fluxes on unlimited slopes at a contact).
template <int MODEL> __device__ __forceinline__ bool phys_prim(const MPar& P, const float* W) {
    if constexpr (MODEL == MODEL_EULER) {
        return W[0] > 0.0f && W[3] + P.gp1 >= 0.0f;
    } else {
        // p + k >= 0  <=>  p eps + kn >= 0 (eps > 0 for 0 <= z <= 1)
        float omz = 1.0f - W[5];
        float eps = W[5] * P.i1 + omz * P.i2, kn = W[5] * P.c1 + omz * P.c2;
        // all six tests evaluated (no short-circuit branches): 2 % faster
        return (W[0] >= 0.0f) & (W[1] >= 0.0f) & (W[0] + W[1] > 0.0f) & (W[5] >= 0.0f) &
               (W[5] <= 1.0f) & (W[4] * eps + kn >= 0.0f);
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

// Limited slopes of all components, d = limit(W - Wm, Wp - W), with the
// limiter chosen once for the cell rather than once per component.
template <int NV>
__device__ __forceinline__ void limit_all(int lim, const float* Wm, const float* W, const float* Wp,
                                          float* d) {
    switch (lim) {
        case LIM_VANLEER:
#pragma unroll
            for (int q = 0; q < NV; ++q) d[q] = limit_f(LIM_VANLEER, W[q] - Wm[q], Wp[q] - W[q]);
            break;
        case LIM_MC:
#pragma unroll
            for (int q = 0; q < NV; ++q) d[q] = limit_f(LIM_MC, W[q] - Wm[q], Wp[q] - W[q]);
            break;
        case LIM_UNLIMITED:
#pragma unroll
            for (int q = 0; q < NV; ++q) d[q] = limit_f(LIM_UNLIMITED, W[q] - Wm[q], Wp[q] - W[q]);
            break;
        default:
#pragma unroll
            for (int q = 0; q < NV; ++q) d[q] = limit_f(LIM_MINMOD, W[q] - Wm[q], Wp[q] - W[q]);
    }
}

// Sound speed of a primitive state.
template <int MODEL> __device__ __forceinline__ float sound_f(const MPar& P, const float* W) {
    if constexpr (MODEL == MODEL_EULER) {
        return fsqrt(fmaxf_s(0.0f, fdiv(P.g1 * (W[3] + P.p1), W[0])));
    } else {
        // c^2 = (k + p (1/eps + 1)) / rho = (kn + p (1 + eps)) / (eps rho)
        float omz = 1.0f - W[5];
        float eps = W[5] * P.i1 + omz * P.i2, kn = W[5] * P.c1 + omz * P.c2;
        float rho = W[0] + W[1];
        return fsqrt(fmaxf_s(0.0f, fdiv(kn + W[4] * (1.0f + eps), eps * rho)));
    }
}

// Half-step evolution X = (0.5 dt/dx) A(W) d (primitive Jacobian).
template <int MODEL>
__device__ __forceinline__ void jac_f(const MPar& P, const float* W, const float* d, float s,
                                      float* X) {
    float c = sound_f<MODEL>(P, W);
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
__device__ __forceinline__ void hllc_prim(const MPar& P, const float* WL, const float* WR,
                                          float* F) {
    using T = ModelTraits<MODEL>;
    constexpr int NV = T::NV;
    float rL, rR, uL, uR, pL, pR, cL, cR, epsL = 1.f, kL = 0.f, epsR = 1.f, kR = 0.f;
    if constexpr (MODEL == MODEL_EULER) {
        rL = WL[0]; uL = WL[1]; pL = WL[3];
        rR = WR[0]; uR = WR[1]; pR = WR[3];
        cL = fsqrt(fmaxf_s(0.0f, fdiv(P.g1 * (pL + P.p1), rL)));
        cR = fsqrt(fmaxf_s(0.0f, fdiv(P.g1 * (pR + P.p1), rR)));
    } else {
        rL = WL[0] + WL[1]; uL = WL[2]; pL = WL[4];
        rR = WR[0] + WR[1]; uR = WR[2]; pR = WR[4];
        mix_f(P, WL[5], epsL, kL);
        mix_f(P, WR[5], epsR, kR);
        cL = fsqrt(fmaxf_s(0.0f, fdiv(kL + pL * (frcp(epsL) + 1.0f), rL)));
        cR = fsqrt(fmaxf_s(0.0f, fdiv(kR + pR * (frcp(epsR) + 1.0f), rR)));
    }
    float SL, SR;
    if (MODEL == MODEL_ALLAIRE && P.pvrs()) {
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
    // per-element selects (a pointer to either side would put both in local memory)
    float rho = left ? rL : rR, u = left ? uL : uR, p = left ? pL : pR;
    float Sk = left ? SL : SR, dS = left ? dSL : dSR;
    float wave = left ? fminf_s(0.0f, SL) : fmaxf_s(0.0f, SR);
    float fac = fdiv(dS, Sk - us);
    // conserved state of the selected side
    float U[NV];
    if constexpr (MODEL == MODEL_EULER) {
        float v = left ? WL[2] : WR[2];
        U[0] = rho;
        U[1] = rho * u;
        U[2] = rho * v;
        U[3] = (p + P.gp1) * P.i1 + 0.5f * rho * (u * u + v * v);
    } else {
        float v = left ? WL[3] : WR[3];
        float eps = left ? epsL : epsR, k = left ? kL : kR;
        U[0] = left ? WL[0] : WR[0];
        U[1] = left ? WL[1] : WR[1];
        U[2] = rho * u;
        U[3] = rho * v;
        U[4] = (p + k) * eps + 0.5f * rho * (u * u + v * v);
        U[5] = left ? WL[5] : WR[5];
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

// The planes of one state buffer of a member, held in registers: the stores
// of a sweep go through pointers the compiler cannot tell apart from the
// member descriptor, so reading the descriptor's pointers again after every
// store would cost a global load each time.
struct MPlanes {
    float4 *v4, *c4;  // components 0-3: value, compensation
    float2 *v2, *c2;  // Allaire E, z: value, compensation
};

template <int MODEL>
__device__ __forceinline__ MPlanes mplanes(const Inst& I, int buf) {
    MPlanes q;
    q.v4 = I.q4[buf][0];
    q.c4 = I.q4[buf][1];
    q.v2 = MODEL == MODEL_ALLAIRE ? I.q2[buf][0] : nullptr;
    q.c2 = MODEL == MODEL_ALLAIRE ? I.q2[buf][1] : nullptr;
    return q;
}

template <int MODEL> __device__ __forceinline__ void load_cell(const MPlanes& Q, long long off, float* h,
                                                               float* l) {
    float4 a = __ldg(Q.v4 + off), b = __ldg(Q.c4 + off);
    h[0] = a.x; h[1] = a.y; h[2] = a.z; h[3] = a.w;
    l[0] = b.x; l[1] = b.y; l[2] = b.z; l[3] = b.w;
    if constexpr (MODEL == MODEL_ALLAIRE) {
        float2 c = __ldg(Q.v2 + off), d = __ldg(Q.c2 + off);
        h[4] = c.x; h[5] = c.y;
        l[4] = d.x; l[5] = d.y;
    }
}

template <int MODEL> __device__ __forceinline__ void store_cell(const MPlanes& Q, long long off,
                                                                const float* h, const float* l) {
    Q.v4[off] = make_float4(h[0], h[1], h[2], h[3]);
    Q.c4[off] = make_float4(l[0], l[1], l[2], l[3]);
    if constexpr (MODEL == MODEL_ALLAIRE) {
        Q.v2[off] = make_float2(h[4], h[5]);
        Q.c2[off] = make_float2(l[4], l[5]);
    }
}

template <int MODEL> __device__ __forceinline__ void load_cell(const Inst& I, int buf,
                                                               long long off, float* h, float* l) {
    load_cell<MODEL>(mplanes<MODEL>(I, buf), off, h, l);
}

// The clip of the updated volume fraction to [z_min, 1 - z_min] on a
// compensated z (value h, compensation l).
__device__ __forceinline__ void clip_z(const Inst& I, float& h, float& l) {
    const double zm = __ldg(&I.z_min);
    const float zlo = (float)zm, zhi = (float)(1.0 - zm);
    if (h + l < zlo) { h = zlo; l = (float)(zm - (double)zlo); }
    if (h + l > zhi) { h = zhi; l = (float)((1.0 - zm) - (double)zhi); }
}

template <int MODEL> __device__ __forceinline__ void store_cell(const Inst& I, int buf,
                                                                long long off, const float* h,
                                                                const float* l) {
    store_cell<MODEL>(mplanes<MODEL>(I, buf), off, h, l);
}

// Shared-memory vectors: one float4 (+ one float2 for Allaire) per slot.
template <int MODEL> struct SVec {
    float4* v4;
    float2* v2;
    __device__ __forceinline__ void put(int s, const float* x) const {
        v4[s] = make_float4(x[0], x[1], x[2], x[3]);
        if constexpr (MODEL == MODEL_ALLAIRE) v2[s] = make_float2(x[4], x[5]);
    }
    __device__ __forceinline__ void get(int s, float* x) const {
        float4 a = v4[s];
        x[0] = a.x; x[1] = a.y; x[2] = a.z; x[3] = a.w;
        if constexpr (MODEL == MODEL_ALLAIRE) {
            float2 b = v2[s];
            x[4] = b.x; x[5] = b.y;
        }
    }
};

template <int MODEL, int DIR, int TS, int NA>
struct MTile {
    static constexpr int NV = ModelTraits<MODEL>::NV;
    static constexpr int LA = TS + 4;
    static constexpr int NSLOT = LA * NA;
    static constexpr int ST = (DIR == DIR_X) ? 1 : NA;
    static constexpr int VB = (MODEL == MODEL_ALLAIRE) ? 24 : 16;  // bytes of one vector
    static_assert(NSLOT == 256, "one staged cell per thread");
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
    // vectors per slot: value, compensation, W, W+, W-, flux; u*, z*; flags;
    // then the staging area the next tile's cells are copied into
    // (value and compensation, slot = thread)
    static constexpr int STG = (6 * VB * NSLOT + 8 * NSLOT + NSLOT + 15) / 16 * 16;
    static constexpr int SMEM = STG + 2 * VB * NSLOT;
};

// Where a tile lies and whether it is skipped.
struct TileGeom {
    int inst, ltile, a_org, b_org, len, wid, cur;
    bool skip;
};

template <int DIR, int TS, int NA>
__device__ __forceinline__ TileGeom tile_geom(const MixedArgs& A, int tile) {
    const int4* e = reinterpret_cast<const int4*>(A.tiles + tile);
    const int4 e0 = e[0], e1 = e[1];
    TileGeom g;
    g.inst = e0.x;
    g.ltile = e0.y;
    g.a_org = e0.z;
    g.b_org = e0.w;
    g.len = e1.x;
    g.wid = e1.y;
    const DevState* st = A.insts[g.inst].st;
    g.skip = !e1.w || st->done || st->n >= e1.z;
    g.cur = st->cur;
    return g;
}

// Starts copying this thread's staged cell of a tile (the boundary mirror
// of pre_sweep picks the source cell) into its staging slot.
template <int MODEL, int DIR, int TS, int NA>
__device__ __forceinline__ void tile_issue(const MixedArgs& A, const TileGeom& g, char* smem) {
    using Tl = MTile<MODEL, DIR, TS, NA>;
    const Inst& I = A.insts[g.inst];
    int a, b;
    Tl::item(threadIdx.x, 0, Tl::LA, a, b);
    const int ga = g.a_org + a, gb = g.b_org + b;
    int src = ga;
    if (ga < 0) src = -ga - 1;
    else if (ga >= g.len) src = 2 * g.len - 1 - ga;
    src = min(max(src, 0), g.len - 1);
    const int gbs = min(gb, g.wid - 1);
    const long long off =
        (DIR == DIR_X) ? (long long)gbs * I.pitch + src : (long long)src * I.pitch + gbs;
    const int buf = g.cur ^ (DIR == DIR_Y);
    char* stg = smem + Tl::STG;
    const int t = threadIdx.x;
    cp_async16(stg + 16 * t, I.q4[buf][0] + off);
    cp_async16(stg + 16 * (Tl::NSLOT + t), I.q4[buf][1] + off);
    if constexpr (MODEL == MODEL_ALLAIRE) {
        cp_async8(stg + 32 * Tl::NSLOT + 8 * t, I.q2[buf][0] + off);
        cp_async8(stg + 40 * Tl::NSLOT + 8 * t, I.q2[buf][1] + off);
    }
    cp_async_commit();
}

// Per-thread wave-speed maxima and mass sums of the tiles of a run.
struct RAcc {
    float mu, mv;
    double m1, m2;
};

template <int MODEL, int DIR, int TS, int NA>
__device__ __forceinline__ void mixed_tile(const MixedArgs& A, const TileGeom& g, int next_tile,
                                           char* smem, RAcc& racc, TileGeom& s_next,
                                           float* s_coef) {
    using Tl = MTile<MODEL, DIR, TS, NA>;
    using MT = ModelTraits<MODEL>;
    constexpr int NV = MT::NV, LA = Tl::LA, NSLOT = Tl::NSLOT, ST = Tl::ST;
    const int tid = threadIdx.x;
    auto vec = [&](int k) {
        SVec<MODEL> v;
        v.v4 = reinterpret_cast<float4*>(smem + k * Tl::VB * NSLOT);
        v.v2 = reinterpret_cast<float2*>(smem + k * Tl::VB * NSLOT + 16 * NSLOT);
        return v;
    };
    const SVec<MODEL> sH = vec(0), sL = vec(1), sW = vec(2), sP = vec(3), sM = vec(4), sF = vec(5);
    float2* sUZ = reinterpret_cast<float2*>(smem + 6 * Tl::VB * NSLOT);
    unsigned char* sFl = reinterpret_cast<unsigned char*>(smem + 6 * Tl::VB * NSLOT + 8 * NSLOT);

    const Inst& I = A.insts[g.inst];
    const MPar P = load_par(I);
    // CTA-wide values of this tile, made once by thread 0 during P1 (shared
    // memory): the sweep's coefficients and the geometry of the next tile
    if (tid == 0) {
        const double dt = I.st->dt;
        const double h_flux = (DIR == DIR_X) ? I.dx : (I.fix_dy ? I.dy : I.dx);
        const double h_upd = (DIR == DIR_X) ? I.dx : I.dy;
        s_coef[0] = (float)(0.5 * (dt / h_flux));
        s_coef[1] = (float)(dt / h_upd);
        TileGeom t;
        if (next_tile < A.ntiles) {
            t = tile_geom<DIR, TS, NA>(A, next_tile);
        } else {
            t.inst = -1;
            t.skip = true;
        }
        s_next = t;
    }

    // ---- P1: boundary sign, rotation, conversion of the fetched cell -------
    {
        int a, b;
        Tl::item(tid, 0, LA, a, b);
        float h[NV], l[NV];
        cp_async_wait_all();
        {
            const char* stg = smem + Tl::STG;
            const float4 x = *reinterpret_cast<const float4*>(stg + 16 * tid);
            const float4 y = *reinterpret_cast<const float4*>(stg + 16 * (NSLOT + tid));
            h[0] = x.x; h[1] = x.y; h[2] = x.z; h[3] = x.w;
            l[0] = y.x; l[1] = y.y; l[2] = y.z; l[3] = y.w;
            if constexpr (MODEL == MODEL_ALLAIRE) {
                const float2 z = *reinterpret_cast<const float2*>(stg + 32 * NSLOT + 8 * tid);
                const float2 w = *reinterpret_cast<const float2*>(stg + 40 * NSLOT + 8 * tid);
                h[4] = z.x; h[5] = z.y;
                l[4] = w.x; l[5] = w.y;
            }
        }
        const int ga = g.a_org + a;
        const int wall_lo = (DIR == DIR_X) ? 0 : 2;
        const bool neg = (ga < 0 && ((P.flags >> (5 + wall_lo)) & 1)) ||
                         (ga >= g.len && ((P.flags >> (6 + wall_lo)) & 1));
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
        c2p_mixed<MODEL>(I, P, h, l, W);
        sH.put(s, h);
        sL.put(s, l);
        sW.put(s, W);
    }
    __syncthreads();
    // the staging slot is free: start copying this thread's cell of the next tile
    {
        const TileGeom gn = s_next;
        if (!gn.skip) tile_issue<MODEL, DIR, TS, NA>(A, gn, smem);
    }
    const float s_half = s_coef[0];
    const float k_upd = s_coef[1];

    // ---- P2: slopes and evolved face states (primitive) ----------------
    if (!P.godunov() && tid < (LA - 2) * NA) {
        int a, b;
        Tl::item(tid, 1, LA - 2, a, b);
        int s = Tl::slot(a, b);
        float W[NV], Wl[NV], Wr[NV], d[NV], X[NV], Wt[NV];
        sW.get(s, W);
        sW.get(s - ST, Wl);
        sW.get(s + ST, Wr);
        limit_all<NV>(P.limiter(), Wl, W, Wr, d);
        unsigned fl = 0;
#pragma unroll
        for (int k = 0; k < NV; ++k) Wt[k] = W[k] + 0.5f * d[k];
        if (phys_prim<MODEL>(P, Wt)) fl |= 1u;
#pragma unroll
        for (int k = 0; k < NV; ++k) Wt[k] = W[k] - 0.5f * d[k];
        if (phys_prim<MODEL>(P, Wt)) fl |= 2u;
        jac_f<MODEL>(P, W, d, s_half, X);
#pragma unroll
        for (int k = 0; k < NV; ++k) Wt[k] = (W[k] + 0.5f * d[k]) - X[k];
        if (phys_prim<MODEL>(P, Wt)) fl |= 4u;
        sP.put(s, Wt);
#pragma unroll
        for (int k = 0; k < NV; ++k) Wt[k] = (W[k] - 0.5f * d[k]) - X[k];
        if (phys_prim<MODEL>(P, Wt)) fl |= 8u;
        sM.put(s, Wt);
        sFl[s] = (unsigned char)fl;
    }
    __syncthreads();

    // ---- P3: HLLC per face -------------------------------------------------
    if (tid < (TS + 1) * NA) {
        int a, b;
        Tl::item(tid, 2, TS + 1, a, b);
        int sR = Tl::slot(a, b), sL = sR - ST;
        float WL[NV], WR[NV];
        bool first = true;
        if (!P.godunov()) {
            unsigned fL = sFl[sL], fR = sFl[sR];
            // zero slopes evolve to the cell state itself; the first-order
            // fallback uses the cell states too
            if ((fL & 1u) && (fR & 2u) && (fL & 4u) && (fR & 8u)) {
                first = false;
                sP.get(sL, WL);
                sM.get(sR, WR);
            }
        }
        if (first) {
            sW.get(sL, WL);
            sW.get(sR, WR);
        }
        float F[NV + 2];
        hllc_prim<MODEL>(P, WL, WR, F);
        sF.put(sR, F);
        sUZ[sR] = make_float2(F[NV], MODEL == MODEL_ALLAIRE ? F[NV + 1] : 0.0f);
    }
    __syncthreads();

    // ---- P4: compensated update, store, reduce -----------------------------
    float r_mu = 0.0f, r_mv = 0.0f;
    double r_m1 = 0.0, r_m2 = 0.0;
    if (tid < TS * NA) {
        int a, b;
        Tl::item(tid, 2, TS, a, b);
        int ga = g.a_org + a, gb = g.b_org + b;
        if (ga < g.len && gb < g.wid) {
            int s = Tl::slot(a, b);
            float hh[NV], ll[NV];
            sH.get(s, hh);
            sL.get(s, ll);
            {
                float FL[NV], FR[NV];
                sF.get(s, FL);
                sF.get(s + ST, FR);
#pragma unroll
                for (int k = 0; k < NV; ++k) {
                    if (MODEL == MODEL_ALLAIRE && k == 5) continue;
                    comp_add(hh[k], ll[k], k_upd * (FL[k] - FR[k]));
                }
            }
            if constexpr (MODEL == MODEL_ALLAIRE) {
                float2 uzL = sUZ[s], uzR = sUZ[s + ST];
                float usL = uzL.x, usR = uzR.x, zsL = uzL.y, zsR = uzR.y;
                float z = hh[5];
                float dz;
                if (P.godunov()) {
                    float zL = sH.v2[s - ST].y, zR = sH.v2[s + ST].y;
                    dz = -k_upd * ((zR - z) * fminf_s(0.0f, usR) + (z - zL) * fmaxf_s(0.0f, usL));
                } else {
                    dz = -k_upd * ((usR * zsR - usL * zsL) - z * (usR - usL));
                }
                comp_add(hh[5], ll[5], dz);
                clip_z(I, hh[5], ll[5]);
                if (hh[0] < 0.0f) { hh[0] = 0.0f; ll[0] = 0.0f; }
                if (hh[1] < 0.0f) { hh[1] = 0.0f; ll[1] = 0.0f; }
            }
            if (DIR == DIR_Y) {  // rotate back
                float t = hh[MT::IM], tl = ll[MT::IM];
                hh[MT::IM] = -hh[MT::IT]; ll[MT::IM] = -ll[MT::IT];
                hh[MT::IT] = t; ll[MT::IT] = tl;
            }
            float Wn[NV];
            c2p_mixed<MODEL>(I, P, hh, ll, Wn);
            if constexpr (MODEL == MODEL_EULER) {
                // density / energy restore as in the plain form (rare)
                if (!(hh[0] > 1e-12f) || !(Wn[3] + P.gp1 > 0.0f)) {
                    float oh[NV], ol[NV], Wo[NV];  // the cell before the update
                    sH.get(s, oh);
                    sL.get(s, ol);
                    if (DIR == DIR_Y) {
                        float t2 = oh[MT::IM], t2l = ol[MT::IM];
                        oh[MT::IM] = -oh[MT::IT]; ol[MT::IM] = -ol[MT::IT];
                        oh[MT::IT] = t2; ol[MT::IT] = t2l;
                    }
                    c2p_mixed<MODEL>(I, P, oh, ol, Wo);
                    float rho = hh[0] > 1e-12f ? hh[0] : oh[0];
                    float u = Wn[1], v = Wn[2];
                    float p = (Wn[3] + P.gp1 > 0.0f) ? Wn[3] : Wo[3];
                    hh[0] = rho; ll[0] = 0.f;
                    hh[1] = rho * u; ll[1] = 0.f;
                    hh[2] = rho * v; ll[2] = 0.f;
                    hh[3] = (p + P.gp1) * P.i1 + 0.5f * rho * (u * u + v * v); ll[3] = 0.f;
                    Wn[0] = rho;
                    Wn[3] = p;
                }
            }
            long long off = (DIR == DIR_X) ? (long long)gb * I.pitch + ga : (long long)ga * I.pitch + gb;
            store_cell<MODEL>(I, g.cur ^ (DIR == DIR_X), off, hh, ll);
            if (DIR == DIR_Y) {
                float c = sound_f<MODEL>(P, Wn);
                r_mu = fabsf(Wn[MT::IM]) + c;
                r_mv = fabsf(Wn[MT::IT]) + c;
                r_m1 = (double)hh[0] + (double)ll[0];
                if constexpr (MODEL == MODEL_ALLAIRE) r_m2 = (double)hh[1] + (double)ll[1];
            }
        }
    }
    if constexpr (DIR == DIR_Y) {  // this thread's wave speeds and masses
        racc.mu = fmaxf_s(racc.mu, r_mu);  // max of FP32 speeds: exact in FP32
        racc.mv = fmaxf_s(racc.mv, r_mv);
        racc.m1 += r_m1;
        racc.m2 += r_m2;
    }
}

// End of the run of an instance's tiles processed by this CTA (y sweep):
// block-reduce the run's wave speeds and masses into the instance's partial
// slot, count the run's tiles, and let the CTA that completes the count pick
// the instance's dt.  CTA c walks the contiguous tile range
// [c * chunk, (c + 1) * chunk), so it meets an instance (tiles [t0, t0 + n))
// in at most one run, and the CTAs that do are c0 = t0 / chunk ..
// (t0 + n - 1) / chunk: slot c - c0 is written exactly once per sweep.
__device__ __forceinline__ void flush_run(const MixedArgs& A, int inst, int slot, int nslots,
                                          int count, RAcc& racc, double dt) {
    const Inst& I = A.insts[inst];
    DevState* st = I.st;
    __shared__ double red[4][8];
    __shared__ bool is_last;
    const int tid = threadIdx.x;
    double mu = (double)racc.mu, mv = (double)racc.mv, m1 = racc.m1, m2 = racc.m2;
    for (int o = 16; o > 0; o >>= 1) {
        mu = smax(mu, __shfl_down_sync(0xffffffffu, mu, o));
        mv = smax(mv, __shfl_down_sync(0xffffffffu, mv, o));
        m1 += __shfl_down_sync(0xffffffffu, m1, o);
        m2 += __shfl_down_sync(0xffffffffu, m2, o);
    }
    if ((tid & 31) == 0) {
        red[0][tid >> 5] = mu;
        red[1][tid >> 5] = mv;
        red[2][tid >> 5] = m1;
        red[3][tid >> 5] = m2;
    }
    __syncthreads();
    if (tid == 0) {
        mu = red[0][0], mv = red[1][0], m1 = red[2][0], m2 = red[3][0];
        for (int w = 1; w < 8; ++w) {
            mu = smax(mu, red[0][w]);
            mv = smax(mv, red[1][w]);
            m1 += red[2][w];
            m2 += red[3][w];
        }
        double* p = I.partials + 4 * slot;
        p[0] = mu;
        p[1] = mv;
        p[2] = m1;
        p[3] = m2;
        __threadfence();
        unsigned t = atomicAdd(&st->ticket, (unsigned)count);
        is_last = (t + (unsigned)count == (unsigned)I.tiles_y);
    }
    __syncthreads();
    if (is_last) {
        __threadfence();
        finish_reduction(st, I.partials, nslots, 1, dt, 0);
    }
    racc.mu = racc.mv = 0.0f;
    racc.m1 = racc.m2 = 0.0;
}

// Persistent sweep: a fixed grid of CTAs walks the tile list of every
// instance in the launch; each thread loads its cell of the next tile while
// the current tile is being computed.
// Resident CTAs per SM: 3 for the y sweeps the batch launches (4 would suit
// the Euler x form, which the batch does not launch).
template <int MODEL, int DIR, int TS, int NA>
__global__ void __launch_bounds__(256, (MODEL == MODEL_EULER && DIR == DIR_X) ? 4 : 3)
    mixed_sweep_kernel(MixedArgs A) {
    extern __shared__ __align__(16) char msm[];
    __shared__ TileGeom s_next;
    __shared__ float s_coef[2];
    const int t_begin = blockIdx.x * A.chunk;
    const int t_end = min(t_begin + A.chunk, A.ntiles);
    if (t_begin >= t_end) return;
    TileGeom g = tile_geom<DIR, TS, NA>(A, t_begin);
    if (!g.skip) tile_issue<MODEL, DIR, TS, NA>(A, g, msm);
    RAcc racc{0.0f, 0.0f, 0.0, 0.0};
    int run_first = t_begin, run_count = 0;
    for (int tile = t_begin; tile < t_end; ++tile) {
        int next = tile + 1 < t_end ? tile + 1 : A.ntiles;  // A.ntiles: none
        const int inst = g.inst;
        TileGeom gn;
        gn.inst = -1;
        gn.skip = true;
        if (!g.skip) {
            mixed_tile<MODEL, DIR, TS, NA>(A, g, next, msm, racc, s_next, s_coef);
            ++run_count;
            gn = s_next;
        } else if (next < A.ntiles) {
            gn = tile_geom<DIR, TS, NA>(A, next);
            if (!gn.skip) tile_issue<MODEL, DIR, TS, NA>(A, gn, msm);
        }
        bool run_ends = next >= A.ntiles || gn.inst != inst;
        if (DIR == DIR_Y && run_ends && run_count > 0) {
            int t0 = run_first - A.tiles[run_first].local;  // first tile of the instance
            int c0 = t0 / A.chunk;
            int nslots = (t0 + A.insts[inst].tiles_y - 1) / A.chunk - c0 + 1;
            flush_run(A, inst, (int)blockIdx.x - c0, nslots, run_count, racc,
                      A.insts[inst].st->dt);
        }
        if (run_ends) {
            run_count = 0;
            run_first = next;
        }
        g = gn;
        __syncthreads();  // shared memory is reused by the next tile
    }
    cp_async_wait_all();
}

}  // namespace mixed
}  // namespace cfd
