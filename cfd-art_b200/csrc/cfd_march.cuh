// Barrier-free warp forms of the mixed-precision sweeps.
//
// Marching strips (the y sweep): a warp owns a strip of 32 lines x A.rows
// cells along the sweep of one instance: lane = line, and every lane walks
// along its line one cell at a time, carrying the window the stencil needs
// from one row to the next in registers (primitive states, the face state,
// the flux).  The rows ahead of the one being computed are copied global ->
// shared with cp.async, three rows in flight, so no registers are held by
// the loads, and each row stays in shared memory until the update that
// starts from it.  The strip length is chosen per launch on the
// host (kMarchMinRows..kMarchMaxRows) so that the strips fill the resident
// warps.  No barrier is needed, and only the two halo cells at each end of
// a strip are re-read.  In the y sweep the lanes are 32 consecutive columns,
// so every step reads 32 consecutive cells (coalesced).  The code also has
// the x form (lanes on 32 rows, each lane reading consecutive cells of its
// row step by step), but on B200 that form measured 1.9x slower than the
// tiled x sweep, so the batch marches in y only.  The arithmetic of every
// cell, face and update is the one of the tiled sweep (cfd_mixed.cuh): the
// same functions in the same order, so the two give the same results bit for
// bit and the autotuner may pick either.
//
// Reduction: each strip reduces its lanes' wave speeds and masses into its
// own slot of the instance's partials; the strip that completes the
// instance's ticket count combines the slots in slot order (reproducible
// sums) and picks the instance's dt.
//
// Warp segments (the x sweep, further down): the lanes hold 32 consecutive
// cells of a row and exchange neighbour values by shuffles.
#pragma once

#include "cfd_mixed.cuh"

namespace cfd {
namespace mixed {

constexpr int kMarchMaxRows = 64, kMarchMinRows = 16;  // rows of a strip (its width is one warp)

// y-sweep frame: the boundary sign of a mirrored row, then (u, v) -> (v, -u).
template <int MODEL>
__device__ __forceinline__ void march_rotate_in(float* h, float* l, bool neg) {
    using MT = ModelTraits<MODEL>;
    if (neg) {
        h[MT::IT] = -h[MT::IT];
        l[MT::IT] = -l[MT::IT];
    }
    float t = h[MT::IM], tl = l[MT::IM];
    h[MT::IM] = h[MT::IT];
    l[MT::IM] = l[MT::IT];
    h[MT::IT] = -t;
    l[MT::IT] = -tl;
}

// Sweep frame of a loaded cell: the boundary sign of a mirrored cell (normal
// momentum), and in y the rotation (u, v) -> (v, -u).
template <int MODEL, int DIR>
__device__ __forceinline__ void march_frame_in(float* h, float* l, bool neg) {
    using MT = ModelTraits<MODEL>;
    if (DIR == DIR_Y) {
        march_rotate_in<MODEL>(h, l, neg);
    } else if (neg) {
        h[MT::IM] = -h[MT::IM];
        l[MT::IM] = -l[MT::IM];
    }
}

// Last-strip finish of the wave-speed reduction, by one warp: slots in slot
// order per lane, then a fixed shuffle tree (reproducible sums).
__device__ __forceinline__ void march_finish(DevState* st, const double* partials, int nslots,
                                             double dt_used) {
    const int lane = threadIdx.x & 31;
    double mu = 0.0, mv = 0.0, m1 = 0.0, m2 = 0.0;
    for (int b = lane; b < nslots; b += 32) {
        mu = smax(mu, __ldcg(partials + 4 * b + 0));
        mv = smax(mv, __ldcg(partials + 4 * b + 1));
        m1 += __ldcg(partials + 4 * b + 2);
        m2 += __ldcg(partials + 4 * b + 3);
    }
    for (int o = 16; o > 0; o >>= 1) {
        mu = smax(mu, __shfl_down_sync(0xffffffffu, mu, o));
        mv = smax(mv, __shfl_down_sync(0xffffffffu, mv, o));
        m1 += __shfl_down_sync(0xffffffffu, m1, o);
        m2 += __shfl_down_sync(0xffffffffu, m2, o);
    }
    if (lane == 0) {
        DevState s = *st;
        s.t = s.t + dt_used;
        s.n = s.n + 1;
        if (fabs(s.t - s.T) < 1e-12) s.t = s.T;
        s.maxu = mu;
        s.maxv = mv;
        s.mass1 = m1 * s.dx * s.dy;
        s.mass2 = m2 * s.dx * s.dy;
        s.dt = choose_dt(s, mu, mv);
        s.done = !(s.t < s.T);
        s.ticket = 0;
        *st = s;
        __threadfence();
    }
}

// Rows staged through shared memory with cp.async (no registers held by the
// loads in flight): a ring of kMSlots slots per lane holding rows k-2 .. k+3
// while row k is computed; kMAhead rows in flight, row k + kMAhead issued
// into the slot of row k - 3 once row k has arrived; per slot MU 16-byte
// units per lane (value and compensation words of components 0-3; for
// Allaire E and z with their compensation words).  The raw cells of row
// k-2, which its update starts from, are therefore read again from the
// ring rather than carried in registers for two rows: 124 -> 115 registers
// for Euler and 5 % less time per y sweep; Allaire's carried window (face
// state, flux) then fits in its 128 registers, where it had to sit in
// shared memory before.
constexpr int kMAhead = 3, kMSlots = kMAhead + 3;
template <int MODEL>
__host__ __device__ constexpr int march_units() {
    return MODEL == MODEL_ALLAIRE ? 3 : 2;
}

// Dynamic shared memory of a 4-warp marching CTA: the staging rings.
template <int MODEL>
__host__ __device__ constexpr int march_smem_bytes() {
    return 4 * kMSlots * march_units<MODEL>() * 32 * 16;
}

// Starts copying the cell at element offset `off` of the planes `Q` (value
// and compensation words) into slot `s` of this lane's staging ring `stg`.
template <int MODEL>
__device__ __forceinline__ void mstage_issue(char* stg, int s, const MPlanes& Q, long long off) {
    constexpr int MU = march_units<MODEL>();
    cp_async16(stg + ((s * MU + 0) * 32) * 16, Q.v4 + off);
    cp_async16(stg + ((s * MU + 1) * 32) * 16, Q.c4 + off);
    if constexpr (MODEL == MODEL_ALLAIRE) {
        cp_async8(stg + ((s * MU + 2) * 32) * 16, Q.v2 + off);
        cp_async8(stg + ((s * MU + 2) * 32) * 16 + 8, Q.c2 + off);
    }
}

// The cell staged in slot `s` (as stored: no mirror, no rotation).
template <int MODEL>
__device__ __forceinline__ void mstage_read(const char* stg, int s, float* h, float* l) {
    constexpr int MU = march_units<MODEL>();
    const float4 a = *reinterpret_cast<const float4*>(stg + ((s * MU + 0) * 32) * 16);
    const float4 b = *reinterpret_cast<const float4*>(stg + ((s * MU + 1) * 32) * 16);
    h[0] = a.x; h[1] = a.y; h[2] = a.z; h[3] = a.w;
    l[0] = b.x; l[1] = b.y; l[2] = b.z; l[3] = b.w;
    if constexpr (MODEL == MODEL_ALLAIRE) {
        const float4 e = *reinterpret_cast<const float4*>(stg + ((s * MU + 2) * 32) * 16);
        h[4] = e.x; h[5] = e.y;
        l[4] = e.z; l[5] = e.w;
    }
}

// One strip: cells [r0, r1) along the sweep of lines [b_org, b_org + 32) of
// instance g.inst ("row" below means a position along the sweep).
template <int MODEL, int DIR>
__device__ __forceinline__ void march_strip(const MixedArgs& A, const TileGeom& g) {
    using MT = ModelTraits<MODEL>;
    constexpr int NV = MT::NV;
    const int lane = threadIdx.x & 31;
    const Inst& I = A.insts[g.inst];
    const MPar P = load_par(I);
    DevState* st = I.st;
    const double dt = st->dt;
    const double h_flux = DIR == DIR_X ? I.dx : (I.fix_dy ? I.dy : I.dx);
    const float s_half = (float)(0.5 * (dt / h_flux));
    const float k_upd = (float)(dt / (DIR == DIR_X ? I.dx : I.dy));
    const int ny = g.len, nx = g.wid;  // cells along the sweep, lines
    const int col = g.b_org + lane;    // this lane's line
    const bool live = col < nx;
    const int c = min(col, nx - 1);
    const int r0 = g.a_org + 2;
    const int r1 = min(r0 + A.rows, ny);
    // the x sweep reads the current buffer, the y sweep the x sweep's output
    const int bin = DIR == DIR_X ? g.cur : g.cur ^ 1, bout = bin ^ 1;
    // Euler holds the planes in registers (2 % faster); Allaire, at its
    // 128-register limit, spilled that way and measured 3 % slower, so it
    // reads them from the member descriptor where it uses them
    const MPlanes qin_r = mplanes<MODEL>(I, bin), qout_r = mplanes<MODEL>(I, bout);
    auto qin = [&] {
        if constexpr (MODEL == MODEL_EULER) return qin_r;
        else return mplanes<MODEL>(I, bin);
    };
    auto qout = [&] {
        if constexpr (MODEL == MODEL_EULER) return qout_r;
        else return mplanes<MODEL>(I, bout);
    };
    const long long pitch = I.pitch;
    const int wall_bit = DIR == DIR_X ? 5 : 7;  // walls L, R / B, T
    const bool wall_lo = (P.flags >> wall_bit) & 1, wall_hi = (P.flags >> (wall_bit + 1)) & 1;
    const bool god = P.godunov();
    const int lim = P.limiter();

    // the mirrored source row of input row k and its sign
    auto src_row = [&](int k, bool& neg) {
        neg = false;
        int r = k;
        if (k < 0) {
            r = -k - 1;
            neg = wall_lo;
        } else if (k >= ny) {
            r = 2 * ny - 1 - k;
            neg = wall_hi;
        }
        return min(max(r, 0), ny - 1);
    };

    float W1[NV], W2[NV];       // W(k-1), W(k-2)
    unsigned flp = 0;           // physicality flags of row k-2
    float Pp[NV], Fl[NV];       // state at the high face of row k-2, flux at its low face
    float us_low = 0.f, zs_low = 0.f;
    float z3 = 0.f;             // z of row k-3 (first-order z update)
    float rmu = 0.f, rmv = 0.f;
    double rm1 = 0.0, rm2 = 0.0;
#pragma unroll
    for (int q = 0; q < NV; ++q) W1[q] = W2[q] = Pp[q] = Fl[q] = 0.f;

    // rows staged ahead (y sweep: line = column, along = row)
    extern __shared__ __align__(16) char march_stage[];
    constexpr int MU = march_units<MODEL>();
    char* stg = march_stage + (threadIdx.x >> 5) * (kMSlots * MU * 32 * 16) +
                16 * lane;
    auto issue = [&](int s, int k) {
        bool ng;
        mstage_issue<MODEL>(stg, s, qin(), (long long)src_row(k, ng) * pitch + c);
    };
    auto staged = [&](int s, float* h, float* l) { mstage_read<MODEL>(stg, s, h, l); };
#pragma unroll
    for (int j = 0; j < kMAhead; ++j) {
        if (r0 - 2 + j <= r1 + 1) issue(j, r0 - 2 + j);
        cp_async_commit();
    }
    int slot = 0;

    for (int k = r0 - 2; k <= r1 + 1; ++k) {
        float h[NV], l[NV];
        bool neg;
        src_row(k, neg);
        asm volatile("cp.async.wait_group %0;\n" ::"n"(kMAhead - 1) : "memory");
        staged(slot, h, l);
        // row k + kMAhead into the slot of row k - 3 (read three rows ago)
        if (k + kMAhead <= r1 + 1) issue(slot >= 3 ? slot - 3 : slot + kMSlots - 3, k + kMAhead);
        cp_async_commit();
        const int slot2 = slot >= 2 ? slot - 2 : slot + kMSlots - 2;  // row k - 2
        slot = slot == kMSlots - 1 ? 0 : slot + 1;
        march_frame_in<MODEL, DIR>(h, l, neg);
        float W0[NV];
        c2p_mixed<MODEL>(I, P, h, l, W0);

        // slopes and evolved face states of row k-1
        float Pn[NV], Mn[NV];
        unsigned fln = 0;
        if (k >= r0 && !god) {
            float d[NV], X[NV];
            limit_all<NV>(lim, W2, W1, W0, d);
#pragma unroll
            for (int q = 0; q < NV; ++q) Pn[q] = W1[q] + 0.5f * d[q];
            if (phys_prim<MODEL>(P, Pn)) fln |= 1u;
#pragma unroll
            for (int q = 0; q < NV; ++q) Pn[q] = W1[q] - 0.5f * d[q];
            if (phys_prim<MODEL>(P, Pn)) fln |= 2u;
            jac_f<MODEL>(P, W1, d, s_half, X);
#pragma unroll
            for (int q = 0; q < NV; ++q) Pn[q] = (W1[q] + 0.5f * d[q]) - X[q];
            if (phys_prim<MODEL>(P, Pn)) fln |= 4u;
#pragma unroll
            for (int q = 0; q < NV; ++q) Mn[q] = (W1[q] - 0.5f * d[q]) - X[q];
            if (phys_prim<MODEL>(P, Mn)) fln |= 8u;
        }

        // HLLC at the face between rows k-2 and k-1
        float Fh[NV + 2];
        if (k >= r0 + 1) {
            float WL[NV], WR[NV];
            const bool second = !god && (flp & 1u) && (fln & 2u) && (flp & 4u) && (fln & 8u);
#pragma unroll
            for (int q = 0; q < NV; ++q) {
                WL[q] = second ? Pp[q] : W2[q];
                WR[q] = second ? Mn[q] : W1[q];
            }
            hllc_prim<MODEL>(P, WL, WR, Fh);
        }

        // compensated update of row k-2
        if (k >= r0 + 2) {
            const int row = k - 2;  // inside [r0, r1): no mirror, no sign
            float hh[NV], ll[NV];
            staged(slot2, hh, ll);  // row k-2 as loaded (inside: no mirror)
            march_frame_in<MODEL, DIR>(hh, ll, false);
#pragma unroll
            for (int q = 0; q < NV; ++q) {
                if (MODEL == MODEL_ALLAIRE && q == 5) continue;
                comp_add(hh[q], ll[q], k_upd * (Fl[q] - Fh[q]));
            }
            if constexpr (MODEL == MODEL_ALLAIRE) {
                const float usL = us_low, usR = Fh[NV], zsL = zs_low, zsR = Fh[NV + 1];
                const float z = hh[5];
                float dz;
                if (god)
                    dz = -k_upd * ((W1[5] - z) * fminf_s(0.0f, usR) + (z - z3) * fmaxf_s(0.0f, usL));
                else
                    dz = -k_upd * ((usR * zsR - usL * zsL) - z * (usR - usL));
                comp_add(hh[5], ll[5], dz);
                clip_z(I, hh[5], ll[5]);
                if (hh[0] < 0.0f) { hh[0] = 0.0f; ll[0] = 0.0f; }
                if (hh[1] < 0.0f) { hh[1] = 0.0f; ll[1] = 0.0f; }
            }
            if (DIR == DIR_Y) {  // rotate back
                float t = hh[MT::IM], tl = ll[MT::IM];
                hh[MT::IM] = -hh[MT::IT];
                ll[MT::IM] = -ll[MT::IT];
                hh[MT::IT] = t;
                ll[MT::IT] = tl;
            }
            float Wn[NV];
            c2p_mixed<MODEL>(I, P, hh, ll, Wn);
            if constexpr (MODEL == MODEL_EULER) {
                // density / energy restore as in the plain form (rare)
                if (!(hh[0] > 1e-12f) || !(Wn[3] + P.gp1 > 0.0f)) {
                    float oh[NV], ol[NV], Wo[NV];  // the cell before the update
                    load_cell<MODEL>(qin(), DIR == DIR_Y ? (long long)row * pitch + c : (long long)c * pitch + row,
                                     oh, ol);
                    c2p_mixed<MODEL>(I, P, oh, ol, Wo);  // stored (unrotated) frame
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
            if (live) {
                store_cell<MODEL>(qout(),
                                  DIR == DIR_Y ? (long long)row * pitch + c
                                               : (long long)c * pitch + row,
                                  hh, ll);
            }
            if (DIR == DIR_Y && live) {
                float cs = sound_f<MODEL>(P, Wn);
                rmu = fmaxf_s(rmu, fabsf(Wn[MT::IM]) + cs);
                rmv = fmaxf_s(rmv, fabsf(Wn[MT::IT]) + cs);
                rm1 += (double)hh[0] + (double)ll[0];
                if constexpr (MODEL == MODEL_ALLAIRE) rm2 += (double)hh[1] + (double)ll[1];
            }
        }

        // shift the window
        if constexpr (MODEL == MODEL_ALLAIRE) z3 = W2[5];
#pragma unroll
        for (int q = 0; q < NV; ++q) {
            W2[q] = W1[q];
            W1[q] = W0[q];
            Pp[q] = Pn[q];
        }
        flp = fln;
        if (k >= r0 + 1) {
#pragma unroll
            for (int q = 0; q < NV; ++q) Fl[q] = Fh[q];
            us_low = Fh[NV];
            zs_low = MODEL == MODEL_ALLAIRE ? Fh[NV + 1] : 0.f;
        }
    }

    if (DIR == DIR_X) return;  // the y sweep reduces
    // this strip's wave speeds and masses into its slot, then the ticket
    double mu = (double)rmu, mv = (double)rmv;
    for (int o = 16; o > 0; o >>= 1) {
        mu = smax(mu, __shfl_down_sync(0xffffffffu, mu, o));
        mv = smax(mv, __shfl_down_sync(0xffffffffu, mv, o));
        rm1 += __shfl_down_sync(0xffffffffu, rm1, o);
        rm2 += __shfl_down_sync(0xffffffffu, rm2, o);
    }
    unsigned ticket = 0;
    if (lane == 0) {
        double* p = I.partials + 4 * g.ltile;
        p[0] = mu;
        p[1] = mv;
        p[2] = rm1;
        p[3] = rm2;
        __threadfence();
        ticket = atomicAdd(&st->ticket, 1u);
    }
    ticket = __shfl_sync(0xffffffffu, ticket, 0);
    if (ticket + 1u == (unsigned)I.tiles_y) {
        __threadfence();
        march_finish(st, I.partials, I.tiles_y, dt);
    }
}

// Persistent sweep: warp w of the W warps of the grid walks the strips w,
// w + W, w + 2W, ... of the launch's strip list, so the strips of members
// that have finished (skipped) are spread over all warps instead of idling
// some of them.
template <int MODEL, int DIR>
__global__ void __launch_bounds__(128) mixed_march_kernel(MixedArgs A) {
    const int gw = blockIdx.x * (blockDim.x >> 5) + (threadIdx.x >> 5);
    const int nw = gridDim.x * (blockDim.x >> 5);
    for (int tile = gw; tile < A.ntiles; tile += nw) {
        const TileGeom g = tile_geom<DIR, kMarchMaxRows, 32>(A, tile);
        if (!g.skip) march_strip<MODEL, DIR>(A, g);
    }
}

// ---- x sweep by warp segments ------------------------------------------------
// A warp owns a tile of kSegCells columns x A.rows rows and walks its rows:
// the 32 lanes hold 32 consecutive cells of a row (kSegCells outputs plus a
// 2-cell halo at each end), so every load and store is coalesced, and the
// neighbours each stencil step needs (primitive states, face states, fluxes)
// come from the adjacent lanes by warp shuffles: no barrier, and shared
// memory only for the rows staged ahead.  The arithmetic is the tiled
// sweep's, in the same order.
// Euler's rows are staged like the marching strips' (kMAhead in flight), in
// a ring of kSSlots slots per lane: the slot refilled at row r is the one
// read at row r - 1 (x sweep 0.255 -> 0.241 ms at 4096^2; the kernel had
// waited on its one-row register prefetch).  Allaire's x sweep is bound by
// instruction issue rather than load latency, and the staging instructions
// made it 4 % slower, so it prefetches the next row into registers.
template <int MODEL>
__host__ __device__ constexpr bool seg_staged() {
    return MODEL == MODEL_EULER;
}
constexpr int kSSlots = kMAhead + 1;
template <int MODEL>
__host__ __device__ constexpr int seg_smem_bytes() {
    return seg_staged<MODEL>() ? 4 * kSSlots * march_units<MODEL>() * 32 * 16 : 0;  // 4 warps per CTA
}
constexpr int kSegCells = 28;  // outputs per row segment
// rows of a tile: chosen per launch on the host (kSegMinRows..kSegRows) so
// that the tiles fill the resident warps
constexpr int kSegRows = 32, kSegMinRows = 12;

template <int N>
__device__ __forceinline__ void shfl_up_n(const float* x, float* y) {
#pragma unroll
    for (int q = 0; q < N; ++q) y[q] = __shfl_up_sync(0xffffffffu, x[q], 1);
}
template <int N>
__device__ __forceinline__ void shfl_down_n(const float* x, float* y) {
#pragma unroll
    for (int q = 0; q < N; ++q) y[q] = __shfl_down_sync(0xffffffffu, x[q], 1);
}

template <int MODEL>
__device__ __forceinline__ void segment_tile(const MixedArgs& A, const TileGeom& g) {
    using MT = ModelTraits<MODEL>;
    constexpr int NV = MT::NV;
    const int lane = threadIdx.x & 31;
    const Inst& I = A.insts[g.inst];
    const MPar P = load_par(I);
    const double dt = I.st->dt;
    const float s_half = (float)(0.5 * (dt / I.dx));
    const float k_upd = (float)(dt / I.dx);
    const int nx = g.len, ny = g.wid;
    const int bin = g.cur, bout = g.cur ^ 1;
    const MPlanes qin = mplanes<MODEL>(I, bin), qout = mplanes<MODEL>(I, bout);
    const long long pitch = I.pitch;
    const bool god = P.godunov();
    const int lim = P.limiter();
    // this lane's column and its mirrored source (pre_sweep's fill)
    const int ga = g.a_org + lane;
    int src = ga;
    bool neg = false;
    if (ga < 0) {
        src = -ga - 1;
        neg = (P.flags >> 5) & 1;
    } else if (ga >= nx) {
        src = 2 * nx - 1 - ga;
        neg = (P.flags >> 6) & 1;
    }
    src = min(max(src, 0), nx - 1);
    const bool writer = lane >= 2 && lane < 2 + kSegCells && ga < nx;
    const int row_end = min(g.b_org + A.rows, ny);

    constexpr bool staged = seg_staged<MODEL>();
    extern __shared__ __align__(16) char seg_stage[];
    constexpr int MU = march_units<MODEL>();
    char* stg = seg_stage + (threadIdx.x >> 5) * (kSSlots * MU * 32 * 16) + 16 * lane;
    float nh[NV], nl[NV];  // the next row (unstaged form)
    if constexpr (staged) {
#pragma unroll
        for (int j = 0; j < kMAhead; ++j) {
            if (g.b_org + j < row_end)
                mstage_issue<MODEL>(stg, j, qin, (long long)(g.b_org + j) * pitch + src);
            cp_async_commit();
        }
    } else {
        load_cell<MODEL>(qin, (long long)g.b_org * pitch + src, nh, nl);
    }
    int slot = 0;
    for (int row = g.b_org; row < row_end; ++row) {
        float h[NV], l[NV];
        if constexpr (staged) {
            asm volatile("cp.async.wait_group %0;\n" ::"n"(kMAhead - 1) : "memory");
            mstage_read<MODEL>(stg, slot, h, l);
            if (row + kMAhead < row_end)
                mstage_issue<MODEL>(stg, slot == 0 ? kSSlots - 1 : slot - 1, qin,
                                    (long long)(row + kMAhead) * pitch + src);
            cp_async_commit();
            slot = slot == kSSlots - 1 ? 0 : slot + 1;
        } else {
#pragma unroll
            for (int q = 0; q < NV; ++q) {
                h[q] = nh[q];
                l[q] = nl[q];
            }
            if (row + 1 < row_end) load_cell<MODEL>(qin, (long long)(row + 1) * pitch + src, nh, nl);
        }
        if (neg) {
            h[MT::IM] = -h[MT::IM];
            l[MT::IM] = -l[MT::IM];
        }
        float W[NV], Wl[NV], Wr[NV];
        c2p_mixed<MODEL>(I, P, h, l, W);
        shfl_up_n<NV>(W, Wl);
        shfl_down_n<NV>(W, Wr);

        // slopes and evolved face states of this cell (used by lanes 1..30)
        float Pf[NV], Mf[NV];
        unsigned fl = 0;
        if (!god) {
            float d[NV], X[NV];
            limit_all<NV>(lim, Wl, W, Wr, d);
#pragma unroll
            for (int q = 0; q < NV; ++q) Pf[q] = W[q] + 0.5f * d[q];
            if (phys_prim<MODEL>(P, Pf)) fl |= 1u;
#pragma unroll
            for (int q = 0; q < NV; ++q) Pf[q] = W[q] - 0.5f * d[q];
            if (phys_prim<MODEL>(P, Pf)) fl |= 2u;
            jac_f<MODEL>(P, W, d, s_half, X);
#pragma unroll
            for (int q = 0; q < NV; ++q) Pf[q] = (W[q] + 0.5f * d[q]) - X[q];
            if (phys_prim<MODEL>(P, Pf)) fl |= 4u;
#pragma unroll
            for (int q = 0; q < NV; ++q) Mf[q] = (W[q] - 0.5f * d[q]) - X[q];
            if (phys_prim<MODEL>(P, Mf)) fl |= 8u;
        } else {
#pragma unroll
            for (int q = 0; q < NV; ++q) Pf[q] = Mf[q] = W[q];
        }

        // HLLC at this cell's low face (between the lane below and this one)
        float PL[NV];
        shfl_up_n<NV>(Pf, PL);
        const unsigned flL = __shfl_up_sync(0xffffffffu, fl, 1);
        float F[NV + 2];
        {
            float WL[NV], WR[NV];
            const bool second = !god && (flL & 1u) && (fl & 2u) && (flL & 4u) && (fl & 8u);
#pragma unroll
            for (int q = 0; q < NV; ++q) {
                WL[q] = second ? PL[q] : Wl[q];
                WR[q] = second ? Mf[q] : W[q];
            }
            hllc_prim<MODEL>(P, WL, WR, F);
        }
        float FR[NV + 2];  // Euler's update needs only the NV fluxes, not u*
        shfl_down_n<MODEL == MODEL_EULER ? NV : NV + 2>(F, FR);

        // compensated update (lanes 2 .. 2 + kSegCells - 1)
#pragma unroll
        for (int q = 0; q < NV; ++q) {
            if (MODEL == MODEL_ALLAIRE && q == 5) continue;
            comp_add(h[q], l[q], k_upd * (F[q] - FR[q]));
        }
        if constexpr (MODEL == MODEL_ALLAIRE) {
            const float usL = F[NV], usR = FR[NV], zsL = F[NV + 1], zsR = FR[NV + 1];
            const float z = h[5];
            float dz;
            if (god)
                dz = -k_upd * ((Wr[5] - z) * fminf_s(0.0f, usR) + (z - Wl[5]) * fmaxf_s(0.0f, usL));
            else
                dz = -k_upd * ((usR * zsR - usL * zsL) - z * (usR - usL));
            comp_add(h[5], l[5], dz);
            clip_z(I, h[5], l[5]);
            if (h[0] < 0.0f) { h[0] = 0.0f; l[0] = 0.0f; }
            if (h[1] < 0.0f) { h[1] = 0.0f; l[1] = 0.0f; }
        }
        if constexpr (MODEL == MODEL_EULER) {
            float Wn[NV];
            c2p_mixed<MODEL>(I, P, h, l, Wn);
            // density / energy restore as in the plain form (rare)
            if (writer && (!(h[0] > 1e-12f) || !(Wn[3] + P.gp1 > 0.0f))) {
                float oh[NV], ol[NV], Wo[NV];  // the cell before the update
                load_cell<MODEL>(qin, (long long)row * pitch + src, oh, ol);
                c2p_mixed<MODEL>(I, P, oh, ol, Wo);
                float rho = h[0] > 1e-12f ? h[0] : oh[0];
                float u = Wn[1], v = Wn[2];
                float p = (Wn[3] + P.gp1 > 0.0f) ? Wn[3] : Wo[3];
                h[0] = rho; l[0] = 0.f;
                h[1] = rho * u; l[1] = 0.f;
                h[2] = rho * v; l[2] = 0.f;
                h[3] = (p + P.gp1) * P.i1 + 0.5f * rho * (u * u + v * v); l[3] = 0.f;
            }
        }
        if (writer) store_cell<MODEL>(qout, (long long)row * pitch + ga, h, l);
    }
}

// Persistent x sweep: warp w of the W warps of the grid walks the tiles w,
// w + W, w + 2W, ... of the launch's tile list.  Euler is bounded to 64
// registers for 8 CTAs per SM (8 % faster than 7 CTAs when the next row was
// still prefetched into registers); Allaire is fastest unbounded.
template <int MODEL>
__global__ void __launch_bounds__(128, MODEL == MODEL_EULER ? 8 : 1)
    mixed_segment_x_kernel(MixedArgs A) {
    const int gw = blockIdx.x * (blockDim.x >> 5) + (threadIdx.x >> 5);
    const int nw = gridDim.x * (blockDim.x >> 5);
    for (int tile = gw; tile < A.ntiles; tile += nw) {
        const TileGeom g = tile_geom<DIR_X, kSegCells, kSegRows>(A, tile);
        if (!g.skip) segment_tile<MODEL>(A, g);
    }
}

}  // namespace mixed
}  // namespace cfd
